// FE_Q(1) variant of the fused tile kernel: one thread per hex cell (or per
// column of two).
//
// Same tiles (8 x 4 x 4 cells), node bricks, work lists, tensor maps, launch
// schedules and arithmetic as tile_kernel<1, ...> in tile_kernel.cuh, but a
// Q1 cell's 8 nodes and 8 Gauss points fit one thread: the sum-factorized
// interpolation, the per-point physics and the integration stay in that
// thread's registers, so the level and flux exchanges of the Q2 layout (and
// their barriers) disappear. A warp is one 8 x 4 layer of cells; nodes shared
// in x and y are summed with shuffles, nodes shared in z through one
// shared-memory exchange, the one CTA barrier per tile. Bricks are
// triple-buffered so that the next-but-one brick can be requested at that
// barrier.
//
// The arithmetic restates source/ThermalOperator.templates.hh:227-751 and
// source/MaterialProperty.hh:529-846 of the reference (adamantine v1.1.9).
#pragma once

#include "tile_kernel.cuh"

namespace adm
{

// CZ cells per thread, stacked in z (1 or 2): with 2, a thread merges the
// node level its two cells share in registers and pays the per-item work
// (prefetch, waits, the barrier, the write-out bookkeeping) once for both.
template <int CZ>
struct Q1Cell
{
  static constexpr int TX = 8, TY = 4, TZ = 4;
  static constexpr int NCELL = TX * TY * TZ;
  static constexpr int NT = NCELL / CZ; // threads: one per column of CZ cells
  static constexpr int NPZ = TZ / CZ;   // thread layers (warps) in z
  static constexpr int MINB = CZ == 1 ? 3 : 4; // resident CTAs per SM the register budget targets (12 or 8 warps)
  static constexpr int BXP = TD<1>::BXP, BY = TD<1>::BY, BZ = TD<1>::BZ;
  static constexpr int BRICKP = (BXP * BY * BZ + 15) / 16 * 16;
  static constexpr int NBUF = 3;
  // dynamic shared memory: NBUF staged bricks and the z-shared node sums
  // [2][4][NT] (one set per item parity)
  static constexpr size_t SMEM = sizeof(double) * (NBUF * BRICKP + 2 * 4 * NT);
  static_assert(TX == TD<1>::TX && TY == TD<1>::TY && TZ == TD<1>::TZ,
                "the Q1 cell kernel uses the tiles of the Q1 tile kernel");
  static_assert(TZ % CZ == 0, "whole cell columns per thread");
};

// Does the tile (tix, tiy, tiz) meet the support of any source of a member
// whose current beam states are `beams` (exact: it skips only points where
// every source is zero by its own cutoff rules)?
template <int TX, int TY, int TZ>
__device__ __forceinline__ bool tile_meets_source(KernelArgs const &args, BeamState const *beams, int n_beams,
                                                  int tix, int tiy, int tiz)
{
  double const x0 = args.origin[0] + TX * tix * args.h[0];
  double const y0 = args.origin[1] + TY * tiy * args.h[1];
  double const z0 = args.origin[2] + TZ * tiz * args.h[2];
  double const x1 = x0 + TX * args.h[0], y1 = y0 + TY * args.h[1], z1 = z0 + TZ * args.h[2];
  bool hit = false;
  for (int b = 0; b < n_beams; ++b)
  {
    BeamState const &bs = beams[b];
    if (!bs.on)
      continue;
    if (bs.type == 2)
    {
      if (x1 >= bs.cube_min[0] && x0 <= bs.cube_max[0] && y1 >= bs.cube_min[1] && y0 <= bs.cube_max[1] &&
          z1 >= bs.cube_min[2] && z0 <= bs.cube_max[2])
        hit = true;
      continue;
    }
    if ((z1 - bs.center[2]) + bs.depth < 0.0)
      continue;
    double const qx = fmin(fmax(bs.center[0], x0), x1);
    double const qy = fmin(fmax(bs.center[1], y0), y1);
    double const dx = qx - bs.center[0], dy = qy - bs.center[1];
    if (dx * dx + dy * dy > bs.five_r2 * (1.0 + 1e-9))
      continue;
    hit = true;
  }
  return hit;
}

// One FE_Q(1) cell of a tile (cell lx, ly, lz of the tile whose first cell
// is ncx0, ncy0, ncz0; info / cur_pmode / cur_pu its prefetched cell data):
// gather the 8 nodes from the staged brick, interpolate to the 8 Gauss
// points, evaluate the physics (straight-line when every point is cold, the
// out-of-line pass otherwise), integrate back, add the face terms, write the
// cell's liquid sum and powder-storage switch. res[e] (e = i + 2 j + 4 k)
// receives the cell's node results, zero when it is inactive or its brick
// did not arrive.
template <int NS, int P, bool FC>
__device__ __forceinline__ void q1_cell(SmemPhys const &sp, MemberData const &md, KernelArgs const &args,
                                        double const *brick, int lx, int ly, int lz, int ncx0, int ncy0,
                                        int ncz0, uint32_t info, int cur_pmode, double cur_pu, bool arrived,
                                        bool do_src, double *res)
{
  constexpr int BXP = TD<1>::BXP, BY = TD<1>::BY;
  MaterialDesc const *gm = md.mat;
  int const cx = ncx0 + lx, cy = ncy0 + ly, cz = ncz0 + lz;
  bool const in_domain = cx < args.nc[0] && cy < args.nc[1] && cz < args.nc[2];
  size_t const c = in_domain ? cx + (size_t)args.nc[0] * (cy + (size_t)args.nc[1] * cz) : 0;
  bool const active = arrived && (info & CI_ACTIVE) != 0;
  int const mat = (info >> CI_MAT_SHIFT) & 15;
#pragma unroll
  for (int e = 0; e < 8; ++e)
    res[e] = 0.0;
  double liq = 0.0;
  uint32_t cmask = 0;
  int pmode = 0;
  double pu = 0.0;
  if (active)
  {
    // nodes (i, j, k) of the cell, e = i + 2 j + 4 k; Gauss points
    // q = qa + 2 qb + 4 qc
    double T[8];
    {
      double u[8], w1[8], w2[8];
#pragma unroll
      for (int e = 0; e < 8; ++e)
        u[e] = brick[(lx + (e & 1)) + BXP * ((ly + ((e >> 1) & 1)) + BY * (lz + (e >> 2)))];
#pragma unroll
      for (int jk = 0; jk < 4; ++jk)
#pragma unroll
        for (int qa = 0; qa < 2; ++qa)
          w1[qa + 2 * jk] = row_dot<1, M_S>(args.S, qa, &u[2 * jk], 1);
#pragma unroll
      for (int qa = 0; qa < 2; ++qa)
#pragma unroll
        for (int k = 0; k < 2; ++k)
#pragma unroll
          for (int qb = 0; qb < 2; ++qb)
            w2[qa + 2 * qb + 4 * k] = row_dot<1, M_S>(args.S, qb, &w1[qa + 4 * k], 2);
#pragma unroll
      for (int ab = 0; ab < 4; ++ab)
#pragma unroll
        for (int qc = 0; qc < 2; ++qc)
          T[ab + 4 * qc] = row_dot<1, M_S>(args.S, qc, &w2[ab], 4);
    }

    if (NS == 3)
    {
      pmode = cur_pmode;
      if (pmode == 1)
        pu = cur_pu;
    }
    double cs = 1.0, sn = 0.0;
    if (sp.has_rotation)
    {
      cs = md.cosv[c];
      sn = md.sinv[c];
    }
    bool const fast_ok = !sp.use_table && sp.isotropic && !sp.has_rotation;
    // below the solidus a cell whose powder ratio is uniformly 0 or 1 is in
    // one pure state: `cold` names it (or -1)
    double const solidus = sp.props[mat][Q_SOLIDUS];
    int cold = -1;
    if (fast_ok)
    {
      if (NS < 3 || pmode == 0)
        cold = 0;
      else if (pmode == 1 && pu == 1.0)
        cold = 2;
    }
    constexpr int PS = kMaxStates * kMaxPoly; // stride between properties
    bool all_cold = cold >= 0;
    if (NS > 1)
    {
#pragma unroll
      for (int q = 0; q < 8; ++q)
        all_cold &= T[q] < solidus;
    }
    // r: the test-function values at the Gauss points -- the fluxes after
    // the collocation D^T in x, y and z, and the source term -- before
    // the S^T back to the nodes
    double r[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
      r[q] = 0.0;
    if (all_cold)
    {
      double const *cold_c = &sp.poly[mat][0][cold][0];
      double crho[P + 1], ccp[P + 1], ck[P + 1];
#pragma unroll
      for (int k = 0; k <= P; ++k)
      {
        crho[k] = cold_c[P_DENSITY * PS + k];
        ccp[k] = cold_c[P_SPECIFIC_HEAT * PS + k];
        ck[k] = cold_c[P_KX * PS + k];
      }
      // cf = -k / (rho c_p) at the points
      double cf[8];
#pragma unroll
      for (int q = 0; q < 8; ++q)
      {
        double const Tq = T[q];
        double const inv = recip(horner_fixed<P>(crho, Tq) * horner_fixed<P>(ccp, Tq));
        cf[q] = -inv * horner_fixed<P>(ck, Tq);
      }
      // Q1 structure (checked on the host): the collocation derivative of
      // the two Gauss points is one row repeated, D[q] = (-d, d), and all
      // eight points weigh 1/8 (cw[q] the same for every q). So along a
      // direction both points of a pair (i0, i1) see the gradient
      // d (T1 - T0), and the D^T of their fluxes adds t to the test value
      // of i1 and -t to that of i0, with
      // t = d^2 cw_d (T1 - T0) (cf_0 + cf_1).
      double const d = args.D[0][1];
      double const K[3] = {d * d * args.cw[0][0], d * d * args.cw[0][1], d * d * args.cw[0][2]};
#pragma unroll
      for (int dir = 0; dir < 3; ++dir)
      {
        int const stride = 1 << dir; // point index step along the direction
#pragma unroll
        for (int p = 0; p < 4; ++p)
        {
          // the pair's first point: p's two bits fill the other directions
          int const lo = p & ((1 << dir) - 1), hi = p >> dir;
          int const i0 = lo + (hi << (dir + 1)), i1 = i0 + stride;
          double const t = (K[dir] * (T[i1] - T[i0])) * (cf[i0] + cf[i1]);
          r[i1] += t;
          r[i0] -= t;
        }
      }
      if (do_src)
      {
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
          int const qa = q & 1, qb = (q >> 1) & 1, qc = q >> 2;
          double const Tq = T[q];
          double const inv = recip(horner_fixed<P>(crho, Tq) * horner_fixed<P>(ccp, Tq));
          double const px = (args.origin[0] + cx * args.h[0]) + args.qx[qa] * args.h[0];
          double const py = (args.origin[1] + cy * args.h[1]) + args.qx[qb] * args.h[1];
          double const pz = (args.origin[2] + cz * args.h[2]) + args.qx[qc] * args.h[2];
          r[q] += beam_sum(sp, px, py, pz) * inv * args.cw[q][3];
        }
      }
    }
    else
    {
      // mixed states, the mushy range, tables, anisotropy or rotation: the
      // out-of-line pass of the Q1 tile kernel, one Gauss-point level at a
      // time, on copies of the level's arrays
#pragma unroll
      for (int qc = 0; qc < 2; ++qc)
      {
        double tq_l[4], az_l[4], axy_l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
          tq_l[i] = T[i + 4 * qc];
          az_l[i] = row_dot<1, M_D>(args.D, qc, &T[i], 4);
          axy_l[i] = 0.0;
        }
        double lacc = 0.0;
        uint32_t cm = 0;
        general_level<1, NS, P>(sp, gm, md, args, mat, qc, cold, pmode, pu, c * 8 + (size_t)4 * qc, cs, sn,
                                fast_ok, do_src, cx, cy, cz, tq_l, az_l, axy_l, &lacc, &cm);
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
          r[i + 4 * qc] += axy_l[i];
#pragma unroll
          for (int m = 0; m < 2; ++m)
            r[i + 4 * m] = entry_mac<1, M_D>(args.D, qc, m, az_l[i], r[i + 4 * m]);
        }
        liq += lacc;
        cmask |= cm << (4 * qc);
      }
    }
    // S^T in z, y and x back to the nodes
    double r1[8], r2[8];
#pragma unroll
    for (int ab = 0; ab < 4; ++ab)
#pragma unroll
      for (int k = 0; k < 2; ++k)
        r1[ab + 4 * k] = col_dot<1, M_S>(args.S, k, &r[ab], 4);
#pragma unroll
    for (int qa = 0; qa < 2; ++qa)
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
          r2[qa + 2 * j + 4 * k] = col_dot<1, M_S>(args.S, j, &r1[qa + 4 * k], 2);
#pragma unroll
    for (int jk = 0; jk < 4; ++jk)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        res[i + 2 * jk] = col_dot<1, M_S>(args.S, i, &r2[2 * jk], 1);

    // convective / radiative faces (face_local_apply,
    // source/ThermalOperator.templates.hh:619-751), per node level
    if (FC && ((info >> CI_FACE_SHIFT) & 63u))
    {
#pragma unroll
      for (int lev = 0; lev < 2; ++lev)
      {
        double fo[4];
        face_terms<1, NS>(sp, gm, md, args, brick, lx, ly, lz, lev, info, mat, c, fo);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          res[e + 4 * lev] += fo[e];
      }
    }
    // state write-back: the liquid sum (read only by the state queries,
    // which see the last evaluation: written by a vmult and by a step's
    // last stage) and, when a point of a uniform powder cell changed, the
    // switch to per-point storage
    if (NS > 1 && (args.mode != 2 || args.last))
      md.liquid_sum[c] = liq;
    if (NS == 3 && pmode != 2 && cmask)
    {
      md.powder_mode[c] = 2;
#pragma unroll
      for (int e = 0; e < 8; ++e)
        if (!((cmask >> e) & 1u))
          md.powder_q[c * 8 + e] = pu;
    }
  }

}

// The persistent loop over work items (as in tile_kernel): CTA b processes
// items b, b + grid, ... (or one contiguous run with args.blocked).
// Per item and thread (the column of CZ cells lx, ly, CZ pz .. CZ pz + CZ - 1
// of the tile): each cell's 8 nodes to its 8 Gauss points, the physics and
// back (q1_cell), then the shared nodes merged and written out. One CTA barrier per
// item (before the z-shared node sums are read); per-item shared state that
// a thread still finishing the previous item may read (roles, the source
// flag, the z sums) alternates between two copies by item parity, and the
// brick of item k + 2 is requested after the barrier of item k into the
// buffer that item k - 1 used.
template <int NS, int P, int SC, bool FC, int CZ>
__global__ void __launch_bounds__(Q1Cell<CZ>::NT, Q1Cell<CZ>::MINB)
    cell_kernel_q1(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ KernelArgs args, int n_items)
{
  using Q = Q1Cell<CZ>;
  constexpr int TX = Q::TX, TY = Q::TY, TZ = Q::TZ, NT = Q::NT, NPZ = Q::NPZ;
  constexpr int NV = 4 * (CZ + 1); // node results of a thread: CZ + 1 levels of 4
  constexpr int BXP = Q::BXP, BY = Q::BY, BZ = Q::BZ, NBUF = Q::NBUF;
  constexpr unsigned kBoxBytes = sizeof(double) * BXP * BY * BZ;
  extern __shared__ __align__(128) double smem[];
  double *const mbuf0 = smem + NBUF * Q::BRICKP; // [2][4][NT]: z-shared node sums per item parity
  __shared__ SmemPhys sp;
  __shared__ __align__(8) uint64_t bars[NBUF];
  __shared__ int src_flag[2];

  int const tid = threadIdx.x;
  int const lx = tid % TX, ly = (tid / TX) % TY, pz = tid / (TX * TY); // cells CZ pz .. CZ pz + CZ - 1
  int const nt0 = args.nt[0], nt1 = args.nt[1];
  int const pitch = args.pitch, nn1 = args.nn[1];

  auto issue = [&](int b, int item) {
    TileWork const wi = args.work[item];
    int const tix = wi.xyz & 2047u, tiy = (wi.xyz >> 11) & 2047u, tiz = wi.xyz >> 22;
    mbar_arrive_expect_tx(&bars[b], kBoxBytes);
    tma_load_brick(smem + b * Q::BRICKP, &tmap, TX * tix, TY * tiy, TZ * tiz, wi.member, &bars[b]);
  };
  auto source_flag = [&](TileWork const &wk) {
    MemberData const &mk = args.members[wk.member];
    return tile_meets_source<TX, TY, TZ>(args, mk.beam_state, mk.n_beams, (int)(wk.xyz & 2047u),
                                         (int)((wk.xyz >> 11) & 2047u), (int)(wk.xyz >> 22));
  };

  // work distribution as in tile_kernel: dynamic with args.claim (each
  // further item claimed two items ahead), else strided or blocked
  bool const dyn = args.claim != nullptr && !args.blocked;
  __shared__ int claimed[2]; // dynamic: the item after the current one, by item parity
  int first, last, step;
  if (dyn || !args.blocked)
  {
    first = blockIdx.x;
    last = n_items;
    step = gridDim.x;
  }
  else
  {
    int const per = (n_items + (int)gridDim.x - 1) / (int)gridDim.x;
    first = (int)blockIdx.x * per;
    last = min(first + per, n_items);
    step = 1;
  }
  int second = first + step; // the item after the first
  if (tid == 0)
  {
#pragma unroll
    for (int b = 0; b < NBUF; ++b)
      mbar_init(&bars[b], 1);
    fence_mbar_init();
    sp.member = -1;
    if (dyn)
    {
      second = first < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
      claimed[1] = second;
    }
  }
  if (tid < 32 && first < last)
  {
    bool const f = source_flag(args.work[first]);
    if (tid == 0)
      src_flag[0] = f;
  }
  __syncthreads();
  if (tid == 0)
  {
    if (first < last)
      issue(0, first);
    if (second < last)
      issue(1, second);
  }

  // the work item and this thread's cells' data, loaded one item ahead
  TileWork nx_w{0, 0, 0u};
  uint32_t nx_info[CZ];
  int nx_pmode[CZ];
  double nx_pu[CZ];
  auto load_item = [&](int item2) {
    nx_w = args.work[item2];
    MemberData const &mk = args.members[nx_w.member];
    int const kx = TX * (int)(nx_w.xyz & 2047u) + lx, ky = TY * (int)((nx_w.xyz >> 11) & 2047u) + ly;
#pragma unroll
    for (int j = 0; j < CZ; ++j)
    {
      int const kz = TZ * (int)(nx_w.xyz >> 22) + CZ * pz + j;
      nx_info[j] = 0u;
      nx_pmode[j] = 0;
      nx_pu[j] = 0.0;
      if (kx < args.nc[0] && ky < args.nc[1] && kz < args.nc[2])
      {
        size_t const kc = kx + (size_t)args.nc[0] * (ky + (size_t)args.nc[1] * kz);
        nx_info[j] = mk.cell_info[kc];
        if (NS == 3)
        {
          // both loaded unconditionally: a load that waited for the mode
          // would stall the thread here
          nx_pmode[j] = mk.powder_mode[kc];
          nx_pu[j] = mk.powder_cell[kc];
        }
      }
    }
  };
  if (first < last)
    load_item(first);

  int it = 0, buf = 0;
  unsigned phase = 0; // completion parity of the current buffer's barrier
  for (int item = first; item < last; ++it)
  {
    double const *brick = smem + buf * Q::BRICKP;
    double *const mbuf = mbuf0 + (it & 1) * 4 * NT; // [4][NT] of this item's parity
    // the next item (claimed during the previous item, published by its
    // barrier) and, on thread 0, the one after it: claimed here into the
    // slot last read at the start of the previous item, its brick requested
    // after this item's barrier
    int const next = dyn ? claimed[(it + 1) & 1] : item + step;
    int next2 = next + step;
    if (dyn && tid == 0)
    {
      next2 = next < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
      claimed[it & 1] = next2;
    }
    TileWork const w = nx_w;
    uint32_t info[CZ];
    int cur_pmode[CZ];
    double cur_pu[CZ];
#pragma unroll
    for (int j = 0; j < CZ; ++j)
    {
      info[j] = nx_info[j];
      cur_pmode[j] = nx_pmode[j];
      cur_pu[j] = nx_pu[j];
    }
    if (next < last)
    {
      load_item(next);
      if (tid < 32)
      {
        bool const f = source_flag(nx_w);
        if (tid == 0)
          src_flag[(it + 1) & 1] = f;
      }
    }
    MemberData const &md = args.members[w.member];
    int const tile = w.tile;
    int const tix = w.xyz & 2047u, tiy = (w.xyz >> 11) & 2047u, tiz = w.xyz >> 22;
    int const colour = (tix & 1) | ((tiy & 1) << 1) | ((tiz & 1) << 2);
    int const ncx0 = TX * tix, ncy0 = TY * tiy, ncz0 = TZ * tiz; // first cell (and node)
    double *const y = args.y_override ? args.y_override : md.y;
    if (sp.member != w.member)
    {
      load_member_constants<NT>(sp, md, tid);
      __syncthreads();
      if (tid == 0)
        sp.member = w.member;
    }
    if (SC == SC_COLOURED && tid < 27)
      sp.role[it & 1][tid] = node_role(md.tile_nbr[tile], colour, tid % 3, (tid / 3) % 3, tid / 9);
    // wait for this item's brick (bounded); a thread whose wait gave up
    // computes nothing and the vote at the barrier ends the CTA before
    // anything is written
    bool const arrived = mbar_wait(&bars[buf], phase);
    bool const do_src = src_flag[it & 1] != 0;

    // the thread's CZ cells, their node results summed per node level
    double res[NV];
#pragma unroll
    for (int e = 0; e < NV; ++e)
      res[e] = 0.0;
#pragma unroll
    for (int j = 0; j < CZ; ++j)
    {
      double cres[8];
      q1_cell<NS, P, FC>(sp, md, args, brick, lx, ly, CZ * pz + j, ncx0, ncy0, ncz0, info[j], cur_pmode[j],
                         cur_pu[j], arrived, do_src, cres);
#pragma unroll
      for (int e = 0; e < 4; ++e)
      {
        res[e + 4 * j] += cres[e];
        res[e + 4 * (j + 1)] += cres[e + 4];
      }
    }

    // ---- per-node sums: a warp is one 8 x 4 layer of cell columns (lane =
    // lx + 8 ly); nodes shared in x and y go to the lower cell by shuffles,
    // the lowest node level of thread layer pz > 0 to the layer below
    // through shared memory
    unsigned const full = 0xffffffffu;
#pragma unroll
    for (int jk = 0; jk < 2 * (CZ + 1); ++jk)
    {
      double const v = __shfl_down_sync(full, res[2 * jk], 1);
      if (lx < TX - 1)
        res[1 + 2 * jk] += v;
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int k = 0; k <= CZ; ++k)
      {
        double const v = __shfl_down_sync(full, res[i + 4 * k], TX);
        if (ly < TY - 1)
          res[i + 2 + 4 * k] += v;
      }
    if (pz > 0)
    {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        mbuf[e * NT + tid] = res[e];
    }
    if (__syncthreads_or(!arrived))
    {
      if (tid == 0)
      {
        atomicCAS(md.error, 0, (int)DERR_TMA_TIMEOUT);
        // let the late copy, and the one requested for the next item, land
        // before the CTA leaves (bounded as well)
        mbar_wait(&bars[buf], phase);
        if (next < last)
          mbar_wait(&bars[buf == NBUF - 1 ? 0 : buf + 1], buf == NBUF - 1 ? phase ^ 1u : phase);
      }
      return;
    }
    // request the next-but-one brick into the buffer the previous item used
    if (tid == 0 && next2 < last)
    {
      fence_proxy_async();
      issue(buf == 0 ? NBUF - 1 : buf - 1, next2);
    }
    if (pz < NPZ - 1)
    {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        res[e + 4 * CZ] += mbuf[e * NT + tid + TX * TY];
    }

    // ---- write-out of the nodes this thread owns (the lower cell of a
    // shared node owns it)
    int rl[NV], slot[NV];
    size_t gidx[NV];
#pragma unroll
    for (int e = 0; e < NV; ++e)
    {
      int const a = e & 1, b = (e >> 1) & 1, k = e >> 2;
      int const X = lx + a, Y = ly + b, Z = CZ * pz + k;
      int const gx = ncx0 + X, gy = ncy0 + Y, gzn = ncz0 + Z;
      bool const own = (a > 0 || lx == 0) && (b > 0 || ly == 0) && (k > 0 || pz == 0);
      bool const inside = gx < args.nn[0] && gy < nn1 && gzn < args.nn[2];
      int const sx = (X == 0 && tix > 0) ? 1 : ((X == TX && tix < nt0 - 1) ? 2 : 0);
      int const sy = (Y == 0 && tiy > 0) ? 1 : ((Y == TY && tiy < nt1 - 1) ? 2 : 0);
      int const sz = (Z == 0 && tiz > 0) ? 1 : ((Z == TZ && tiz < args.nt[2] - 1) ? 2 : 0);
      slot[e] = 0;
      if constexpr (SC == SC_TWO_PASS)
        rl[e] = (own && inside) ? two_pass_slot<HaloOf<1>>(X, Y, Z, sx, sy, sz, &slot[e]) : 0;
      else
        rl[e] = (own && inside) ? (SC == SC_ATOMIC ? 4 : (sp.role[it & 1][sx + 3 * sy + 9 * sz] | 4)) : 0;
      gidx[e] = gx + (size_t)pitch * (gy + (size_t)nn1 * gzn);
    }
    if constexpr (SC == SC_TWO_PASS)
      write_nodes_two_pass<HaloOf<1>, NV>(args, md, tile, res, rl, gidx, slot);
    else
      write_nodes<SC == SC_ATOMIC, NV>(args, md, y, res, rl, gidx);
    // vmult writes zeros into the row padding of the node layout (the
    // two-pass gather does that itself)
    if (SC == SC_COLOURED && args.mode == 0 && tix == nt0 - 1 && pitch > args.nn[0])
    {
      int const npad = pitch - args.nn[0];
      for (int i = tid; i < npad * BY * BZ; i += NT)
      {
        int const X = i % npad, Y = (i / npad) % BY, Z = i / (npad * BY);
        int const gy = ncy0 + Y, gzn = ncz0 + Z;
        if (gy < nn1 && gzn < args.nn[2])
          args.vdst[args.nn[0] + X + (size_t)pitch * (gy + (size_t)nn1 * gzn)] = 0.0;
      }
    }
    // next buffer of the ring
    if (++buf == NBUF)
    {
      buf = 0;
      phase ^= 1u;
    }
    item = next;
  }
}

// Launches the persistent Q1 cell kernel over n_items work items with at
// most the number of CTAs that are resident at once on the device.
template <int NS, int P, int SC, bool FC, int CZ>
void launch_cell_q1_f(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  using Q = Q1Cell<CZ>;
  static int grid_cap = 0;
  if (grid_cap == 0)
  {
    cudaFuncSetAttribute(cell_kernel_q1<NS, P, SC, FC, CZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Q::SMEM);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cell_kernel_q1<NS, P, SC, FC, CZ>, Q::NT, Q::SMEM);
    grid_cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  int const grid = n_items < grid_cap ? n_items : grid_cap;
  cell_kernel_q1<NS, P, SC, FC, CZ><<<grid, Q::NT, Q::SMEM, stream>>>(map, a, n_items);
}

// ------------------------------------------------------------ column variant
// One warp per CTA and per tile: thread (lx, ly) walks its column of TZ
// cells bottom to top, carrying the node level two cells share in
// registers; a node level is complete when the cell above it is done, and
// it is merged across the warp with shuffles and written out then. The
// warp's tiles need no CTA barrier (a warp vote before the first write and
// __syncwarp for the shared state), so a warp whose tile is slow (cells in
// the mushy range, the source) holds up no other warp; cell data are
// prefetched one cell ahead.
struct Q1Col
{
  static constexpr int TX = 8, TY = 4, TZ = 4;
  static constexpr int NT = TX * TY; // one warp
  static constexpr int MINB = 12;    // resident CTAs (warps) per SM the register budget targets
  static constexpr int BRICKP = Q1Cell<1>::BRICKP;
  static constexpr int NBUF = 3;
  static constexpr size_t SMEM = sizeof(double) * NBUF * BRICKP;
  static_assert(TX == TD<1>::TX && TY == TD<1>::TY && TZ == TD<1>::TZ,
                "the Q1 column kernel uses the tiles of the Q1 tile kernel");
};

template <int NS, int P, int SC, bool FC>
__global__ void __launch_bounds__(Q1Col::NT, Q1Col::MINB)
    cell_kernel_q1_col(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ KernelArgs args,
                       int n_items)
{
  using Q = Q1Col;
  constexpr int TX = Q::TX, TY = Q::TY, TZ = Q::TZ, NT = Q::NT, NBUF = Q::NBUF;
  constexpr int BXP = Q1Cell<1>::BXP, BY = Q1Cell<1>::BY, BZ = Q1Cell<1>::BZ;
  constexpr unsigned kBoxBytes = sizeof(double) * BXP * BY * BZ;
  unsigned const full = 0xffffffffu;
  extern __shared__ __align__(128) double smem[];
  __shared__ SmemPhys sp;
  __shared__ __align__(8) uint64_t bars[NBUF];

  int const lane = threadIdx.x;
  int const lx = lane % TX, ly = lane / TX;
  int const nt0 = args.nt[0], nt1 = args.nt[1];
  int const pitch = args.pitch, nn1 = args.nn[1];

  auto issue = [&](int b, int item) {
    TileWork const wi = args.work[item];
    int const tix = wi.xyz & 2047u, tiy = (wi.xyz >> 11) & 2047u, tiz = wi.xyz >> 22;
    mbar_arrive_expect_tx(&bars[b], kBoxBytes);
    tma_load_brick(smem + b * Q::BRICKP, &tmap, TX * tix, TY * tiy, TZ * tiz, wi.member, &bars[b]);
  };
  // the cell data of cell (lx, ly, kz) of work item wk (zeros outside the mesh)
  auto load_cell = [&](TileWork const &wk, int kz, uint32_t &info, int &pmode, double &pu) {
    MemberData const &mk = args.members[wk.member];
    int const kx = TX * (int)(wk.xyz & 2047u) + lx, ky = TY * (int)((wk.xyz >> 11) & 2047u) + ly;
    int const kzz = TZ * (int)(wk.xyz >> 22) + kz;
    info = 0u;
    pmode = 0;
    pu = 0.0;
    if (kx < args.nc[0] && ky < args.nc[1] && kzz < args.nc[2])
    {
      size_t const kc = kx + (size_t)args.nc[0] * (ky + (size_t)args.nc[1] * kzz);
      info = mk.cell_info[kc];
      if (NS == 3)
      {
        pmode = mk.powder_mode[kc];
        pu = mk.powder_cell[kc];
      }
    }
  };

  // work distribution as in cell_kernel_q1 (dynamic with args.claim, else
  // strided or blocked)
  bool const dyn = args.claim != nullptr && !args.blocked;
  __shared__ int claimed[2];
  int first, last, step;
  if (dyn || !args.blocked)
  {
    first = blockIdx.x;
    last = n_items;
    step = gridDim.x;
  }
  else
  {
    int const per = (n_items + (int)gridDim.x - 1) / (int)gridDim.x;
    first = (int)blockIdx.x * per;
    last = min(first + per, n_items);
    step = 1;
  }
  int second = first + step;
  if (lane == 0)
  {
#pragma unroll
    for (int b = 0; b < NBUF; ++b)
      mbar_init(&bars[b], 1);
    fence_mbar_init();
    sp.member = -1;
    if (dyn)
    {
      second = first < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
      claimed[1] = second;
    }
    if (first < last)
      issue(0, first);
    if (second < last)
      issue(1, second);
  }
  __syncwarp();
  second = __shfl_sync(full, second, 0);

  // the work item (loaded one item ahead) and the cell data of the next
  // cell to compute (one cell ahead)
  TileWork w_cur{0, 0, 0u}, w_next{0, 0, 0u};
  uint32_t nx_info = 0u;
  int nx_pmode = 0;
  double nx_pu = 0.0;
  if (first < last)
  {
    w_cur = args.work[first];
    load_cell(w_cur, 0, nx_info, nx_pmode, nx_pu);
  }

  int it = 0, buf = 0;
  unsigned phase = 0;
  for (int item = first; item < last; ++it)
  {
    double const *brick = smem + buf * Q::BRICKP;
    int const next = dyn ? claimed[(it + 1) & 1] : item + step;
    int next2 = next + step;
    if (dyn && lane == 0)
    {
      next2 = next < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
      claimed[it & 1] = next2;
    }
    next2 = __shfl_sync(full, next2, 0);
    TileWork const w = w_cur;
    if (next < last)
      w_next = args.work[next]; // used by the last cell's prefetch and the next item
    MemberData const &md = args.members[w.member];
    int const tile = w.tile;
    int const tix = w.xyz & 2047u, tiy = (w.xyz >> 11) & 2047u, tiz = w.xyz >> 22;
    int const colour = (tix & 1) | ((tiy & 1) << 1) | ((tiz & 1) << 2);
    int const ncx0 = TX * tix, ncy0 = TY * tiy, ncz0 = TZ * tiz;
    double *const y = args.y_override ? args.y_override : md.y;
    if (sp.member != w.member)
    {
      __syncwarp();
      load_member_constants<NT>(sp, md, lane);
      __syncwarp();
      if (lane == 0)
        sp.member = w.member;
    }
    if (SC == SC_COLOURED && lane < 27)
      sp.role[it & 1][lane] = node_role(md.tile_nbr[tile], colour, lane % 3, (lane / 3) % 3, lane / 9);
    bool const do_src =
        tile_meets_source<TX, TY, TZ>(args, sp.beams, sp.n_beams, tix, tiy, tiz);
    // wait for this item's brick (bounded); if any lane's wait gave up the
    // warp leaves before anything is written
    bool const arrived = mbar_wait(&bars[buf], phase);
    if (__any_sync(full, !arrived))
    {
      if (lane == 0)
      {
        atomicCAS(md.error, 0, (int)DERR_TMA_TIMEOUT);
        mbar_wait(&bars[buf], phase);
        if (next < last)
          mbar_wait(&bars[buf == NBUF - 1 ? 0 : buf + 1], buf == NBUF - 1 ? phase ^ 1u : phase);
      }
      return;
    }
    __syncwarp(); // the roles and member constants are visible to the warp
    // every lane has finished the previous item: its buffer takes the
    // next-but-one brick
    if (lane == 0 && next2 < last)
    {
      fence_proxy_async();
      issue(buf == 0 ? NBUF - 1 : buf - 1, next2);
    }

    double carry[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int k = 0; k <= TZ; ++k)
    {
      double lev[4];
      if (k < TZ)
      {
        uint32_t const info = nx_info;
        int const pmode = nx_pmode;
        double const pu = nx_pu;
        // prefetch the cell above (or the next item's first cell)
        if (k + 1 < TZ)
          load_cell(w, k + 1, nx_info, nx_pmode, nx_pu);
        else if (next < last)
          load_cell(w_next, 0, nx_info, nx_pmode, nx_pu);
        double cres[8];
        q1_cell<NS, P, FC>(sp, md, args, brick, lx, ly, k, ncx0, ncy0, ncz0, info, pmode, pu, true, do_src,
                           cres);
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
          lev[e] = carry[e] + cres[e];
          carry[e] = cres[e + 4];
        }
      }
      else
      {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          lev[e] = carry[e];
      }
      // node level k: x then y neighbours' shares to the lower cell
#pragma unroll
      for (int j = 0; j < 2; ++j)
      {
        double const v = __shfl_down_sync(full, lev[2 * j], 1);
        if (lx < TX - 1)
          lev[1 + 2 * j] += v;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
      {
        double const v = __shfl_down_sync(full, lev[i], TX);
        if (ly < TY - 1)
          lev[i + 2] += v;
      }
      // write-out of the level's nodes this thread owns
      int rl[4], slot[4];
      size_t gidx[4];
      int const Z = k, gzn = ncz0 + Z;
      int const sz = (Z == 0 && tiz > 0) ? 1 : ((Z == TZ && tiz < args.nt[2] - 1) ? 2 : 0);
#pragma unroll
      for (int e = 0; e < 4; ++e)
      {
        int const a = e & 1, b = e >> 1;
        int const X = lx + a, Y = ly + b;
        int const gx = ncx0 + X, gy = ncy0 + Y;
        bool const own = (a > 0 || lx == 0) && (b > 0 || ly == 0);
        bool const inside = gx < args.nn[0] && gy < nn1 && gzn < args.nn[2];
        int const sx = (X == 0 && tix > 0) ? 1 : ((X == TX && tix < nt0 - 1) ? 2 : 0);
        int const sy = (Y == 0 && tiy > 0) ? 1 : ((Y == TY && tiy < nt1 - 1) ? 2 : 0);
        slot[e] = 0;
        if constexpr (SC == SC_TWO_PASS)
          rl[e] = (own && inside) ? two_pass_slot<HaloOf<1>>(X, Y, Z, sx, sy, sz, &slot[e]) : 0;
        else
          rl[e] = (own && inside) ? (SC == SC_ATOMIC ? 4 : (sp.role[it & 1][sx + 3 * sy + 9 * sz] | 4)) : 0;
        gidx[e] = gx + (size_t)pitch * (gy + (size_t)nn1 * gzn);
      }
      if constexpr (SC == SC_TWO_PASS)
        write_nodes_two_pass<HaloOf<1>, 4>(args, md, tile, lev, rl, gidx, slot);
      else
        write_nodes<SC == SC_ATOMIC, 4>(args, md, y, lev, rl, gidx);
    }
    // vmult writes zeros into the row padding of the node layout (the
    // two-pass gather does that itself)
    if (SC == SC_COLOURED && args.mode == 0 && tix == nt0 - 1 && pitch > args.nn[0])
    {
      int const npad = pitch - args.nn[0];
      for (int i = lane; i < npad * BY * BZ; i += NT)
      {
        int const X = i % npad, Y = (i / npad) % BY, Z = i / (npad * BY);
        int const gy = ncy0 + Y, gzn = ncz0 + Z;
        if (gy < nn1 && gzn < args.nn[2])
          args.vdst[args.nn[0] + X + (size_t)pitch * (gy + (size_t)nn1 * gzn)] = 0.0;
      }
    }
    if (++buf == NBUF)
    {
      buf = 0;
      phase ^= 1u;
    }
    w_cur = w_next;
    item = next;
  }
}

template <int NS, int P, int SC, bool FC>
void launch_cell_q1_col_f(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  using Q = Q1Col;
  static int grid_cap = 0;
  if (grid_cap == 0)
  {
    cudaFuncSetAttribute(cell_kernel_q1_col<NS, P, SC, FC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Q::SMEM);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cell_kernel_q1_col<NS, P, SC, FC>, Q::NT, Q::SMEM);
    grid_cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  int const grid = n_items < grid_cap ? n_items : grid_cap;
  cell_kernel_q1_col<NS, P, SC, FC><<<grid, Q::NT, Q::SMEM, stream>>>(map, a, n_items);
}

template <int NS, int P, int SC, int CZ>
void launch_cell_q1_z(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  if (a.faces)
    launch_cell_q1_f<NS, P, SC, true, CZ>(map, a, n_items, stream);
  else
    launch_cell_q1_f<NS, P, SC, false, CZ>(map, a, n_items, stream);
}

// a.cells_per_thread 4: the column variant (one warp per tile), 2: two
// cells per thread (z), else one
template <int NS, int P, int SC>
void launch_cell_q1_s(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  if (a.cells_per_thread == 4)
  {
    if (a.faces)
      launch_cell_q1_col_f<NS, P, SC, true>(map, a, n_items, stream);
    else
      launch_cell_q1_col_f<NS, P, SC, false>(map, a, n_items, stream);
  }
  else if (a.cells_per_thread == 2)
    launch_cell_q1_z<NS, P, SC, 2>(map, a, n_items, stream);
  else
    launch_cell_q1_z<NS, P, SC, 1>(map, a, n_items, stream);
}

// The schedule of a launch: a.atomic, else a.two_pass, else coloured.
template <int NS, int P>
void launch_cell_q1(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  if (a.atomic)
    launch_cell_q1_s<NS, P, SC_ATOMIC>(map, a, n_items, stream);
  else if (a.two_pass)
    launch_cell_q1_s<NS, P, SC_TWO_PASS>(map, a, n_items, stream);
  else
    launch_cell_q1_s<NS, P, SC_COLOURED>(map, a, n_items, stream);
}

} // namespace adm
