// Hand-written adjoint of the explicit time step (no counterpart in the
// reference, which only runs the forward problem).
//
// Objective: J = sum over observation steps n and points p of
// (T_n[node_p] - target_{n,p})^2, T_n the temperature after n steps of the
// configured explicit Runge-Kutta method (source/ThermalPhysics.templates.hh:854-888).
// The gradient with respect to the logarithms of the conductivity scale, the
// specific-heat scale and the source strength comes from the discrete
// adjoint of the forward stages, including the phase history
// s' = min(1 - l(T), s) of every Gauss point:
//   forward stage i: Y_i = y + dt sum_j a_ij k_j,  (k_i, s_{i+1}) = (M^-1 r(Y_i, s_i), s'(Y_i, s_i))
//   step:            y_new = y + dt sum_i b_i k_i
//   adjoint, i = s-1 .. 0:
//     lambda_k_i = dt b_i lambda_y_new + sum_{l > i} dt a_li lambda_Y_l
//     (lambda_Y_i, lambda_s_i) = transpose of stage i applied to (M^-1 lambda_k_i, lambda_s_{i+1})
//   lambda_y = lambda_y_new + sum_i lambda_Y_i
// The forward states are checkpointed every K steps (temperature and the
// sparse powder history) and each K-step segment is recomputed, stage by
// stage, right before its backward sweep.
#include "adjoint_kernel.cuh"
#include "beam_state.cuh"
#include "capi_common.hpp"
#include "../../include/adamantine_b200_adjoint.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace adm
{
namespace
{
template <int DEG, int NS, bool GEN>
void launch_adj(CUtensorMap const &ymap, CUtensorMap const &mmap, AdjArgs const &a, int n_items,
                cudaStream_t stream)
{
  using T_ = TD<DEG>;
  size_t const smem = sizeof(double) * (4 * T_::BRICKP + 4 * T_::NN * T_::NCELL);
  static int grid_cap = 0;
  if (grid_cap == 0)
  {
    ADM_CK(cudaFuncSetAttribute(adjoint_kernel<DEG, NS, GEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    ADM_CK(cudaGetDevice(&dev));
    ADM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ADM_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel<DEG, NS, GEN>, T_::NT, smem));
    grid_cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  int const grid = n_items < grid_cap ? n_items : grid_cap;
  adjoint_kernel<DEG, NS, GEN><<<grid, T_::NT, smem, stream>>>(ymap, mmap, a, n_items);
}

// the backward member data's stage clock
__global__ void bclock_kernel(double *clock, double t, double dt)
{
  if (threadIdx.x == 0)
  {
    clock[0] = t;
    clock[1] = dt;
  }
}

template <bool GEN>
void launch_adjoint_g(int deg, int ns, CUtensorMap const &ym, CUtensorMap const &mm, AdjArgs const &a, int n_items,
                      cudaStream_t stream)
{
  switch (deg * 10 + ns)
  {
  case 11:
    launch_adj<1, 1, GEN>(ym, mm, a, n_items, stream);
    break;
  case 12:
    launch_adj<1, 2, GEN>(ym, mm, a, n_items, stream);
    break;
  case 13:
    launch_adj<1, 3, GEN>(ym, mm, a, n_items, stream);
    break;
  case 21:
    launch_adj<2, 1, GEN>(ym, mm, a, n_items, stream);
    break;
  case 22:
    launch_adj<2, 2, GEN>(ym, mm, a, n_items, stream);
    break;
  case 23:
    launch_adj<2, 3, GEN>(ym, mm, a, n_items, stream);
    break;
  default:
    throw Error(ADM_ERR_INVALID, "no adjoint kernel for this degree / state count");
  }
}

// gen: the variant with rotation, faces and cube sources
void launch_adjoint(int deg, int ns, bool gen, CUtensorMap const &ym, CUtensorMap const &mm, AdjArgs const &a,
                    int n_items, cudaStream_t stream)
{
  if (gen)
    launch_adjoint_g<true>(deg, ns, ym, mm, a, n_items, stream);
  else
    launch_adjoint_g<false>(deg, ns, ym, mm, a, n_items, stream);
}

// resid[p] = y[idx[p]] - target[p]; *J += sum_p resid[p]^2 (one block, fixed
// summation order).
__global__ void misfit_kernel(double const *y, int64_t const *idx, double const *target, int n, double *resid,
                              double *J)
{
  __shared__ double part[256];
  double s = 0.0;
  for (int p = threadIdx.x; p < n; p += blockDim.x)
  {
    double const r = y[idx[p]] - target[p];
    resid[p] = r;
    s += r * r;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if ((int)threadIdx.x < o)
      part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    *J += part[0];
}

// Tile geometry for the activity flags of the backward sweep.
struct TileGrid
{
  int pitch, nn1, deg, t[3], nt[3];
};

// lambda[idx[p]] += 2 resid[p] (points may repeat a node); the tiles that
// hold the node (up to eight) are marked for the next stage.
__global__ void inject_kernel(double *lam, int64_t const *idx, double const *resid, int n, TileGrid g,
                              uint8_t *act)
{
  int const p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n)
    return;
  int64_t const node = idx[p];
  atomicAdd(&lam[node], 2.0 * resid[p]);
  if (!act)
    return;
  int const ni[3] = {(int)(node % g.pitch), (int)((node / g.pitch) % g.nn1), (int)(node / ((int64_t)g.pitch * g.nn1))};
  for (int m = 0; m < 8; ++m)
  {
    int tc[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d)
    {
      int const span = g.deg * g.t[d];
      int c = ni[d] / span;
      if ((m >> d) & 1)
      {
        if (ni[d] % span != 0)
          ok = false;
        c -= 1;
      }
      if (c < 0 || c >= g.nt[d])
        ok = false;
      tc[d] = c;
    }
    if (ok)
      act[tc[0] + (size_t)g.nt[0] * (tc[1] + (size_t)g.nt[1] * tc[2])] = 1;
  }
}


struct LamTerms
{
  double const *v[4];
  double c[4];
  int n;
};

__device__ __forceinline__ double lamk_point(double *mu, double const *inv_mass, double *lam, LamTerms const &pend,
                                             double cb, LamTerms const &t, double *zero, size_t i)
{
  double L = lam[i];
  if (pend.n > 0)
  {
    for (int l = 0; l < pend.n; ++l)
      L += pend.v[l][i];
    lam[i] = L;
  }
  double s = cb * L;
  for (int l = 0; l < t.n; ++l)
    s = fma(t.c[l], t.v[l][i], s);
  double const m = inv_mass[i] * s;
  mu[i] = m;
  zero[i] = 0.0;
  return fabs(m);
}

// lam += sum of the pending stage adjoints of the step after (pend, at the
// first stage of a step), mu = inv_mass * (cb * lam + sum_l c_l lam_Y_l),
// and the stage adjoint the next launch accumulates into is cleared
// (zero, which may be one of the pending vectors: read before written).
// Also, for the stage's transpose launch: the work items of the marked
// tiles (sel, counter n_sel), and the heat-source state at the stage time
// (md, when given); and it clears what the next stage accumulates into: the
// other max and counter slots and the next stage's tile flags.
struct LamkAux
{
  unsigned long long *mu_max, *mu_max_next;
  int *n_sel, *n_sel_next;
  TileWork const *work;
  int n_items;
  uint8_t const *act_cur;
  uint8_t *act_next;
  size_t n_tiles;
  TileWork *sel;
  MemberData *md;
  double c;
};

__global__ void lamk_kernel(double *mu, double const *inv_mass, double *lam, LamTerms pend, double cb, LamTerms t,
                            double *zero, size_t n, LamkAux x)
{
  size_t const i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i == 0)
  {
    *x.mu_max_next = 0ull;
    *x.n_sel_next = 0;
  }
  if (i < x.n_tiles)
    x.act_next[i] = 0;
  if (i < (size_t)x.n_items)
  {
    TileWork const w = x.work[i];
    if (x.act_cur[w.tile])
      x.sel[atomicAdd(x.n_sel, 1)] = w;
  }
  if (x.md && blockIdx.x == 0 && (int)threadIdx.x < x.md->n_beams)
    prepare_beam(*x.md, threadIdx.x, x.c);
  unsigned long long *const mu_max = x.mu_max;
  double m = 0.0;
  if (i < n)
    m = lamk_point(mu, inv_mass, lam, pend, cb, t, zero, i);
  // max |mu| of the stage: warp, block, then one atomic per block (bit
  // patterns of non-negative doubles order as integers)
  __shared__ double wmax[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0)
    wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      m = fmax(m, wmax[w]);
    if (m > 0.0)
      atomicMax(mu_max, (unsigned long long)__double_as_longlong(m));
  }
}

// lam += sum_l lam_Y_l
__global__ void sum_kernel(double *lam, LamTerms t, size_t n)
{
  size_t const i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double s = lam[i];
  for (int l = 0; l < t.n; ++l)
    s += t.v[l][i];
  lam[i] = s;
}

unsigned blocks(size_t n) { return (unsigned)((n + 255) / 256); }
} // namespace

class Adjoint
{
public:
  explicit Adjoint(Thermal &t) : th_(t)
  {
    if (!t.setup_done_)
      throw Error(ADM_ERR_INVALID, "setup() has not been called");
    ADM_CK(cudaSetDevice(t.device_));
    C_ = t.mesh_.n_cells;
    NN_ = (t.mesh_.deg + 1) * (t.mesh_.deg + 1) * (t.mesh_.deg + 1);
    n_ = t.mesh_.n_nodes;
    gen_ = general_kernel();
    NFP_ = face_points();
    save_phase(init_mode_, init_cell_, init_q_, init_face_);
  }

  // the kernel variant with rotation, faces and cube sources is needed
  bool general_kernel() const
  {
    Thermal const &t = th_;
    bool g = t.has_rotation_ || !t.adiabatic_only_;
    for (int b = 0; b < t.cfg_.n_sources; ++b)
      g = g || t.cfg_.sources[b].type == 2;
    return g;
  }

  // values of the face points' powder history (three states with faces)
  size_t face_points() const
  {
    Thermal const &t = th_;
    int const np = t.mesh_.deg + 1;
    return (t.ns_ == 3 && !t.adiabatic_only_) ? (size_t)t.topo_.n_slots * 6 * np * np : 0;
  }

  // The stores and the captured initial phase state are sized by the
  // handle's cells when the adjoint was created: cells activated since then
  // (a new face-point layout, a deposition angle) need a new adjoint.
  void check_handle() const
  {
    if (!th_.setup_done_)
      throw Error(ADM_ERR_INVALID, "the thermal handle is not set up");
    if (face_points() != NFP_ || general_kernel() != gen_)
      throw Error(ADM_ERR_INVALID, "the thermal handle's cells changed after the adjoint was created; create a new "
                                   "adjoint");
  }

  void set_observations(int n_obs_steps, int32_t const *steps, int n_points, int64_t const *index,
                        double const *targets)
  {
    if (n_obs_steps < 0 || n_points < 0 || (n_obs_steps > 0 && (!steps || !targets)) ||
        (n_points > 0 && !index))
      throw Error(ADM_ERR_INVALID, "invalid observation arguments");
    for (int p = 0; p < n_points; ++p)
      if (index[p] < 0 || (size_t)index[p] >= n_)
        throw Error(ADM_ERR_INVALID, "observation node index out of range");
    obs_steps_.assign(steps, steps + n_obs_steps);
    n_points_ = n_points;
    idx_.alloc(std::max(1, n_points));
    tgt_.alloc(std::max<size_t>(1, (size_t)n_obs_steps * n_points));
    resid_.alloc(std::max<size_t>(1, (size_t)n_obs_steps * n_points));
    Jd_.alloc(1);
    if (n_points > 0)
      ADM_CK(cudaMemcpy(idx_.p, index, n_points * sizeof(int64_t), cudaMemcpyHostToDevice));
    if (n_obs_steps > 0 && n_points > 0)
      ADM_CK(cudaMemcpy(tgt_.p, targets, (size_t)n_obs_steps * n_points * sizeof(double),
                        cudaMemcpyHostToDevice));
  }

  // Forward run from the captured initial phase state: J and the final field.
  double objective(double t0, double dt, int n_steps, double const *y0, double *y_final)
  {
    NvtxRange const nvtx_range("adm::adjoint_objective");
    check_run(n_steps, 1);
    forward(t0, dt, n_steps, y0, 0);
    double J = 0.0;
    ADM_CK(cudaMemcpyAsync(&J, Jd_.p, sizeof(double), cudaMemcpyDeviceToHost, th_.stream_));
    if (y_final)
      ADM_CK(cudaMemcpyAsync(y_final, y_.p, n_ * sizeof(double), cudaMemcpyDeviceToDevice, th_.stream_));
    ADM_CK(cudaStreamSynchronize(th_.stream_));
    return J;
  }

  // K <= 0: the longest segment whose stage stores fit in half of the free
  // device memory (every step of the run when it fits: no recompute)
  int auto_interval(int n_steps)
  {
    Thermal &t = th_;
    ADM_CK(cudaSetDevice(t.device_));
    int const S = t.tab_.s;
    double const per_step = 8.0 * S * ((double)n_ + (t.ns_ == 3 ? (double)C_ * NN_ : 0.0) + (double)NFP_);
    size_t free_b = 0, total_b = 0;
    ADM_CK(cudaMemGetInfo(&free_b, &total_b));
    // the stores already held are released before the new ones are made
    double const held = 8.0 * ((double)Ystore_.n + (double)Sstore_.n + (double)Ystore2_.n + (double)Sstore2_.n +
                               (double)Fstore_.n + (double)Fstore2_.n);
    double const budget = 0.5 * ((double)free_b + held);
    double const fit = std::floor(budget / per_step);
    if (fit >= (double)n_steps)
      return n_steps;
    // segments recomputed while the previous one runs backward: two stores
    double const fit2 = std::floor(fit / 2.0);
    if (fit2 < 1.0)
      throw Error(ADM_ERR_ALLOC, "not enough device memory for one step of adjoint stores");
    return (int)fit2;
  }

  int last_interval() const { return last_K_; }

  double gradient(double t0, double dt, int n_steps, int K, double const *y0, double *grad, double *y_final)
  {
    NvtxRange const nvtx_range("adm::adjoint_gradient");
    if (K <= 0 && n_steps >= 1)
      K = auto_interval(n_steps);
    check_run(n_steps, K);
    last_K_ = K;
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    int const S = t.tab_.s;
    // per step of a segment: the S stage inputs and (3 states) S phase
    // states; with more than one segment two stores alternate, so that the
    // recompute of a segment runs while the one after it goes backward
    int const n_seg = (n_steps + K - 1) / K;
    Ystore_.alloc((size_t)K * S * n_);
    if (t.ns_ == 3)
      Sstore_.alloc((size_t)K * S * C_ * NN_);
    if (NFP_)
      Fstore_.alloc((size_t)K * S * NFP_);
    if (n_seg > 1)
    {
      Ystore2_.alloc((size_t)K * S * n_);
      if (t.ns_ == 3)
        Sstore2_.alloc((size_t)K * S * C_ * NN_);
      if (NFP_)
        Fstore2_.alloc((size_t)K * S * NFP_);
    }
    ystore_[0] = Ystore_.p;
    ystore_[1] = n_seg > 1 ? Ystore2_.p : Ystore_.p;
    sstore_[0] = Sstore_.p;
    sstore_[1] = n_seg > 1 ? Sstore2_.p : Sstore_.p;
    fstore_[0] = Fstore_.p;
    fstore_[1] = n_seg > 1 ? Fstore2_.p : Fstore_.p;
    rec_buf_ = (n_seg - 1) & 1;
    forward(t0, dt, n_steps, y0, K);
    double J = 0.0;
    ADM_CK(cudaMemcpyAsync(&J, Jd_.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (y_final)
      ADM_CK(cudaMemcpyAsync(y_final, y_.p, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // final phase state of the forward run, restored at the end
    save_phase(fin_mode_, fin_cell_, fin_q_, fin_face_);

    bool const ns3 = t.ns_ == 3;
    size_t const qn = C_ * NN_;
    lam_.alloc(n_);
    mu_.alloc(n_);
    lamY_.alloc(n_ * S);
    mumax_.alloc(2);
    ADM_CK(cudaMemsetAsync(mumax_.p, 0, 2 * sizeof(unsigned long long), st));
    stage_count_ = 0;
    act_a_.alloc(t.mesh_.n_tiles);
    act_b_.alloc(t.mesh_.n_tiles);
    act_cur_ = act_a_.p;
    act_next_ = act_b_.p;
    ADM_CK(cudaMemsetAsync(act_cur_, 0, t.mesh_.n_tiles, st));
    sel_.alloc(std::max(1, t.colour_off_[8]));
    nsel_.alloc(2);
    ADM_CK(cudaMemsetAsync(nsel_.p, 0, 2 * sizeof(int), st));
    ADM_CK(cudaMemsetAsync(lam_.p, 0, n_ * sizeof(double), st));
    if (ns3)
    {
      ls_a_.alloc(qn);
      ls_b_.alloc(qn);
      ADM_CK(cudaMemsetAsync(ls_a_.p, 0, qn * sizeof(double), st));
      ADM_CK(cudaMemsetAsync(ls_b_.p, 0, qn * sizeof(double), st));
    }
    clear_face_adjoint(st);
    grad_d_.alloc(3);
    ADM_CK(cudaMemsetAsync(grad_d_.p, 0, 3 * sizeof(double), st));
    // the backward sweep runs on its own stream with its own member data
    // (stage clock and beam state: the recompute on the handle's stream
    // writes the handle's); everything else it reads is read-only here
    backward_setup();
    cudaStream_t const bs = bst_;
    ADM_CK(cudaEventRecord(ev_start_, st));
    ADM_CK(cudaStreamWaitEvent(bs, ev_start_, 0));
    ADM_CK(cudaEventRecord(ev_rec_[(n_seg - 1) & 1], st));
    // the stage adjoints of a step are added into lam by the first stage
    // launch of the step before (and once at the end)
    LamTerms all{};
    all.n = S;
    for (int i = 0; i < S; ++i)
      all.v[i] = lamY_.p + (size_t)i * n_;
    bool pending = false;
    for (int seg = n_seg - 1; seg >= 0; --seg)
    {
      int const n0 = seg * K, n1 = std::min(n_steps, n0 + K);
      int const b = seg & 1;
      // the segment's stages are recorded (the forward run recorded the last)
      ADM_CK(cudaStreamWaitEvent(bs, ev_rec_[b], 0));
      double const *ys = ystore_[b];
      double *ss = sstore_[b];
      double const *fs = fstore_[b];
      // backward sweep over the segment
      for (int n = n1 - 1; n >= n0; --n)
      {
        inject(n + 1, bs);
        bclock_kernel<<<1, 32, 0, bs>>>(bclock_.p, times_[n], dt);
        for (int i = S - 1; i >= 0; --i)
        {
          LamTerms lt{};
          lt.n = 0;
          for (int l = i + 1; l < S; ++l)
            if (t.tab_.a[l][i] != 0.0)
            {
              lt.v[lt.n] = lamY_.p + (size_t)l * n_;
              lt.c[lt.n] = dt * t.tab_.a[l][i];
              ++lt.n;
            }
          double *lamYi = lamY_.p + (size_t)i * n_;
          LamTerms pend{};
          pend.n = 0;
          if (i == S - 1 && pending)
            pend = all;
          int const slot = stage_count_ & 1;
          ++stage_count_;
          int const count = t.colour_off_[8];
          LamkAux x{};
          x.mu_max = mumax_.p + slot;
          x.mu_max_next = mumax_.p + (slot ^ 1);
          x.n_sel = nsel_.p + slot;
          x.n_sel_next = nsel_.p + (slot ^ 1);
          x.work = t.awork_d_.p;
          x.n_items = count;
          x.act_cur = act_cur_;
          x.act_next = act_next_;
          x.n_tiles = t.mesh_.n_tiles;
          x.sel = sel_.p;
          x.md = t.cfg_.n_sources > 0 ? bmd_.p : nullptr;
          x.c = t.tab_.c[i];
          size_t const threads = std::max({n_, x.n_tiles, (size_t)count});
          lamk_kernel<<<blocks(threads), 256, 0, bs>>>(mu_.p, t.inv_mass_.p, lam_.p, pend, dt * t.tab_.b[i], lt,
                                                       lamYi, n_, x);
          ADM_CK(cudaGetLastError());
          size_t const rslot = (size_t)(n - n0) * S + i;
          AdjArgs A;
          std::memset(&A, 0, sizeof(A));
          A.k = t.base_args();
          A.k.members = bmd_.p;
          A.yv = ys + rslot * n_;
          A.mu = mu_.p;
          if (ns3)
          {
            A.s_in = ss + rslot * qn;
            A.lam_s_out = ls_a_.p;
            A.lam_s_in = ls_b_.p;
            A.powder_start = init_mode_.p;
          }
          if (NFP_)
          {
            A.sf_in = fs + rslot * NFP_;
            A.lam_sf_out = lsf_a_.p;
            A.lam_sf_in = lsf_b_.p;
          }
          A.lam_y = lamYi;
          A.grad = grad_d_.p;
          A.mu_max = reinterpret_cast<double const *>(x.mu_max);
          A.flush = flush_;
          // visit the marked tiles only; they mark the next stage's
          A.n_items_dev = x.n_sel;
          A.act_next = act_next_;
          run_kernel(A, sel_.p, bs);
          std::swap(act_cur_, act_next_);
          if (ns3)
            std::swap(ls_a_.p, ls_b_.p);
          if (NFP_)
            std::swap(lsf_a_.p, lsf_b_.p);
        }
        pending = true;
      }
      ADM_CK(cudaEventRecord(ev_bwd_[b], bs));
      // meanwhile: recompute the segment before from its checkpoint into the
      // other store, once the backward sweep that last read it has ended
      if (seg >= 1)
      {
        int const nb = b ^ 1, s0 = (seg - 1) * K, s1 = seg * K;
        if (seg + 1 <= n_seg - 1)
          ADM_CK(cudaStreamWaitEvent(st, ev_bwd_[nb], 0));
        ADM_CK(cudaMemcpyAsync(y_.p, ck_y_.p + (size_t)(seg - 1) * n_, n_ * sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
        if (ns3)
          restore_phase(seg - 1);
        rec_buf_ = nb;
        for (int n = s0; n < s1; ++n)
          record_step(n, s0, dt);
        ADM_CK(cudaEventRecord(ev_rec_[nb], st));
      }
    }
    if (pending)
    {
      sum_kernel<<<blocks(n_), 256, 0, bs>>>(lam_.p, all, n_);
      ADM_CK(cudaGetLastError());
    }
    // join the backward stream
    ADM_CK(cudaEventRecord(ev_start_, bs));
    ADM_CK(cudaStreamWaitEvent(st, ev_start_, 0));
    double g[3] = {0, 0, 0};
    ADM_CK(cudaMemcpyAsync(g, grad_d_.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    // the handle ends with the phase state of the forward run
    if (ns3)
    {
      ADM_CK(cudaMemcpyAsync(t.powder_mode_.p, fin_mode_.p, C_, cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(t.powder_cell_.p, fin_cell_.p, C_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(t.powder_q_.p, fin_q_.p, qn * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    if (NFP_)
      ADM_CK(cudaMemcpyAsync(t.face_powder_.p, fin_face_.p, NFP_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaStreamSynchronize(st));
    grad[0] = g[0];
    grad[1] = g[1];
    grad[2] = g[2];
    grad[3] = g[2];
    return J;
  }

  // lambda = (dr/dT)^T mu at the field y with the handle's current phase
  // state held fixed (no powder-history chain): the transpose operator.
  void vmult_transpose(double *lam, double const *y, double const *mu, double *grad)
  {
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    check_handle();
    ADM_CK(cudaSetDevice(t.device_));
    bool const ns3 = t.ns_ == 3;
    size_t const qn = C_ * NN_;
    ADM_CK(cudaMemsetAsync(lam, 0, n_ * sizeof(double), st));
    grad_d_.alloc(3);
    ADM_CK(cudaMemsetAsync(grad_d_.p, 0, 3 * sizeof(double), st));
    t.prepare_stage(0.0);
    AdjArgs A;
    std::memset(&A, 0, sizeof(A));
    A.k = t.base_args();
    A.yv = y;
    A.mu = mu;
    if (ns3)
    {
      ls_a_.alloc(qn);
      ls_b_.alloc(qn);
      Sstore_.alloc(qn);
      ADM_CK(cudaMemsetAsync(ls_a_.p, 0, qn * sizeof(double), st));
      launch_expand_powder(t.cell_info_d_.p, NN_, t.powder_mode_.p, t.powder_cell_.p, t.powder_q_.p, Sstore_.p,
                           C_, st);
      A.s_in = Sstore_.p;
      A.lam_s_out = ls_a_.p;
      A.lam_s_in = ls_b_.p;
    }
    if (NFP_)
    {
      clear_face_adjoint(st);
      A.sf_in = t.face_powder_.p;
      A.lam_sf_out = lsf_a_.p;
      A.lam_sf_in = lsf_b_.p;
    }
    A.lam_y = lam;
    A.grad = grad_d_.p;
    run_kernel(A);
    double g[3];
    ADM_CK(cudaMemcpyAsync(g, grad_d_.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ADM_CK(cudaStreamSynchronize(st));
    if (grad)
      for (int k = 0; k < 3; ++k)
        grad[k] = g[k];
  }

private:
  // one launch over the work items of every colour (atomics merge the nodes
  // that tiles share)
  TileGrid tile_grid() const
  {
    Mesh const &m = th_.mesh_;
    TileGrid g{};
    g.pitch = m.pitch;
    g.nn1 = m.nn[1];
    g.deg = m.deg;
    g.t[0] = m.tx;
    g.t[1] = m.ty;
    g.t[2] = m.tz;
    for (int d = 0; d < 3; ++d)
      g.nt[d] = m.nt[d];
    return g;
  }

  // work: the items to visit (default: every tile of the handle)
  void run_kernel(AdjArgs &A, TileWork const *work = nullptr, cudaStream_t stream = nullptr)
  {
    Thermal &t = th_;
    int const count = t.colour_off_[8];
    if (count == 0)
      return;
    A.k.work = work ? work : t.awork_d_.p;
    CUtensorMap const ym = brick_map(t.mesh_, A.yv, 1, n_);
    CUtensorMap const mm = brick_map(t.mesh_, A.mu, 1, n_);
    launch_adjoint(t.mesh_.deg, t.ns_, gen_, ym, mm, A, count, stream ? stream : t.stream_);
    ADM_CK(cudaGetLastError());
  }

  void check_run(int n_steps, int K)
  {
    if (n_steps < 1)
      throw Error(ADM_ERR_INVALID, "n_steps must be positive");
    if (K < 1)
      throw Error(ADM_ERR_INVALID, "checkpoint interval must be positive");
    for (int s : obs_steps_)
      if (s < 0 || s > n_steps)
        throw Error(ADM_ERR_INVALID, "observation step outside [0, n_steps]");
    check_handle();
    ADM_CK(cudaSetDevice(th_.device_));
  }

  // both face-powder adjoint buffers allocated and zeroed
  void clear_face_adjoint(cudaStream_t st)
  {
    if (!NFP_)
      return;
    lsf_a_.alloc(NFP_);
    lsf_b_.alloc(NFP_);
    ADM_CK(cudaMemsetAsync(lsf_a_.p, 0, NFP_ * sizeof(double), st));
    ADM_CK(cudaMemsetAsync(lsf_b_.p, 0, NFP_ * sizeof(double), st));
  }

  void save_phase(DevBuf<uint8_t> &mode, DevBuf<double> &cell, DevBuf<double> &q, DevBuf<double> &face)
  {
    Thermal &t = th_;
    if (t.ns_ != 3)
      return;
    cudaStream_t const st = t.stream_;
    if (NFP_)
    {
      face.alloc(NFP_);
      ADM_CK(cudaMemcpyAsync(face.p, t.face_powder_.p, NFP_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    mode.alloc(C_);
    cell.alloc(C_);
    q.alloc(C_ * NN_);
    ADM_CK(cudaMemcpyAsync(mode.p, t.powder_mode_.p, C_, cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaMemcpyAsync(cell.p, t.powder_cell_.p, C_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaMemcpyAsync(q.p, t.powder_q_.p, C_ * NN_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }

  void restore_phase(int seg)
  {
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    ADM_CK(cudaMemcpyAsync(t.powder_mode_.p, ck_mode_.p + (size_t)seg * C_, C_, cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaMemcpyAsync(t.powder_cell_.p, ck_cell_.p + (size_t)seg * C_, C_ * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaMemcpyAsync(t.powder_q_.p, ck_q_.p + (size_t)seg * C_ * NN_, C_ * NN_ * sizeof(double),
                           cudaMemcpyDeviceToDevice, st));
    if (NFP_)
      ADM_CK(cudaMemcpyAsync(t.face_powder_.p, ck_face_.p + (size_t)seg * NFP_, NFP_ * sizeof(double),
                             cudaMemcpyDeviceToDevice, st));
  }

  void checkpoint(int seg)
  {
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    ADM_CK(cudaMemcpyAsync(ck_y_.p + (size_t)seg * n_, y_.p, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (t.ns_ == 3)
    {
      ADM_CK(cudaMemcpyAsync(ck_mode_.p + (size_t)seg * C_, t.powder_mode_.p, C_, cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(ck_cell_.p + (size_t)seg * C_, t.powder_cell_.p, C_ * sizeof(double),
                             cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(ck_q_.p + (size_t)seg * C_ * NN_, t.powder_q_.p, C_ * NN_ * sizeof(double),
                             cudaMemcpyDeviceToDevice, st));
    }
    if (NFP_)
      ADM_CK(cudaMemcpyAsync(ck_face_.p + (size_t)seg * NFP_, t.face_powder_.p, NFP_ * sizeof(double),
                             cudaMemcpyDeviceToDevice, st));
  }

  // One step n of the forward run, stage by stage as Thermal::launch_step
  // does it, recording each stage's input field and phase state in slot
  // (n - n0) of the segment store.
  void record_step(int n, int n0, double dt)
  {
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    int const S = t.tab_.s;
    size_t const qn = C_ * NN_;
    t.set_clock(times_[n], dt);
    for (int i = 0; i < S; ++i)
    {
      t.prepare_stage(t.tab_.c[i]);
      KernelArgs a = t.stage_args(i);
      a.y_override = y_.p;
      double const *src = i == 0 ? y_.p : (a.src_sel == 1 ? t.za_p_ : t.zb_p_);
      size_t const slot = (size_t)(n - n0) * S + i;
      ADM_CK(cudaMemcpyAsync(ystore_[rec_buf_] + slot * n_, src, n_ * sizeof(double), cudaMemcpyDeviceToDevice,
                             st));
      if (t.ns_ == 3)
        launch_expand_powder(t.cell_info_d_.p, NN_, t.powder_mode_.p, t.powder_cell_.p, t.powder_q_.p,
                             sstore_[rec_buf_] + slot * qn, C_, st, init_mode_.p);
      if (NFP_)
        ADM_CK(cudaMemcpyAsync(fstore_[rec_buf_] + slot * NFP_, t.face_powder_.p, NFP_ * sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
      t.launch_pass(a, src);
    }
  }

  void observe(int n)
  {
    for (size_t k = 0; k < obs_steps_.size(); ++k)
      if (obs_steps_[k] == n && n_points_ > 0)
      {
        misfit_kernel<<<1, 256, 0, th_.stream_>>>(y_.p, idx_.p, tgt_.p + k * n_points_, n_points_,
                                                  resid_.p + k * n_points_, Jd_.p);
        ADM_CK(cudaGetLastError());
      }
  }

  void inject(int n, cudaStream_t stream)
  {
    for (size_t k = 0; k < obs_steps_.size(); ++k)
      if (obs_steps_[k] == n && n_points_ > 0)
      {
        inject_kernel<<<blocks(n_points_), 256, 0, stream>>>(lam_.p, idx_.p, resid_.p + k * n_points_,
                                                                  n_points_, tile_grid(), act_cur_);
        ADM_CK(cudaGetLastError());
      }
  }

  // Forward run from the initial phase state; K > 0 checkpoints every K steps.
  void forward(double t0, double dt, int n_steps, double const *y0, int K)
  {
    Thermal &t = th_;
    cudaStream_t const st = t.stream_;
    if (obs_steps_.empty() && n_points_ == 0)
      Jd_.alloc(1);
    y_.alloc(n_);
    ADM_CK(cudaMemcpyAsync(y_.p, y0, n_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (t.ns_ == 3)
    {
      ADM_CK(cudaMemcpyAsync(t.powder_mode_.p, init_mode_.p, C_, cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(t.powder_cell_.p, init_cell_.p, C_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
      ADM_CK(cudaMemcpyAsync(t.powder_q_.p, init_q_.p, C_ * NN_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    if (NFP_)
      ADM_CK(cudaMemcpyAsync(t.face_powder_.p, init_face_.p, NFP_ * sizeof(double), cudaMemcpyDeviceToDevice, st));
    ADM_CK(cudaMemsetAsync(Jd_.p, 0, sizeof(double), st));
    if (K > 0)
    {
      int const n_seg = (n_steps + K - 1) / K;
      ck_y_.alloc((size_t)n_seg * n_);
      if (t.ns_ == 3)
      {
        ck_mode_.alloc((size_t)n_seg * C_);
        ck_cell_.alloc((size_t)n_seg * C_);
        ck_q_.alloc((size_t)n_seg * C_ * NN_);
      }
      if (NFP_)
        ck_face_.alloc((size_t)n_seg * NFP_);
    }
    times_.assign(n_steps + 1, 0.0);
    double tt = t0;
    observe(0);
    int const last0 = K > 0 ? ((n_steps - 1) / K) * K : n_steps;
    for (int n = 0; n < n_steps; ++n)
    {
      if (K > 0 && n % K == 0)
        checkpoint(n / K);
      times_[n] = tt;
      if (n >= last0)
      {
        // last segment: record the stages now instead of recomputing them
        record_step(n, last0, dt);
        tt = tt + dt;
      }
      else
        tt = t.evolve_one_time_step(tt, dt, y_.p);
      observe(n + 1);
    }
    times_[n_steps] = tt;
  }

  // the backward stream, its events and member data: a copy of the handle's
  // with its own stage clock and beam state
  void backward_setup()
  {
    Thermal &t = th_;
    if (!bst_)
    {
      ADM_CK(cudaStreamCreateWithFlags(&bst_, cudaStreamNonBlocking));
      ADM_CK(cudaEventCreateWithFlags(&ev_start_, cudaEventDisableTiming));
      for (int i = 0; i < 2; ++i)
      {
        ADM_CK(cudaEventCreateWithFlags(&ev_rec_[i], cudaEventDisableTiming));
        ADM_CK(cudaEventCreateWithFlags(&ev_bwd_[i], cudaEventDisableTiming));
      }
    }
    MemberData md;
    ADM_CK(cudaMemcpyAsync(&md, t.member_d_.p, sizeof(MemberData), cudaMemcpyDeviceToHost, t.stream_));
    ADM_CK(cudaStreamSynchronize(t.stream_));
    bbeam_.alloc(kMaxBeams);
    bclock_.alloc(2);
    md.beam_state = bbeam_.p;
    md.clock = bclock_.p;
    bmd_.alloc(1);
    ADM_CK(cudaMemcpyAsync(bmd_.p, &md, sizeof(MemberData), cudaMemcpyHostToDevice, t.stream_));
    ADM_CK(cudaStreamSynchronize(t.stream_));
  }

public:
  ~Adjoint()
  {
    if (bst_)
    {
      cudaStreamSynchronize(bst_);
      cudaEventDestroy(ev_start_);
      for (int i = 0; i < 2; ++i)
      {
        cudaEventDestroy(ev_rec_[i]);
        cudaEventDestroy(ev_bwd_[i]);
      }
      cudaStreamDestroy(bst_);
    }
  }
  Adjoint(Adjoint const &) = delete;
  Adjoint &operator=(Adjoint const &) = delete;

  // adjoint values at or below flush * (the stage's max |mu|) count as zero
  // (whole tiles of them are skipped)
  double flush_ = 1e-30;
  int last_K_ = 0;

private:
  Thermal &th_;
  size_t C_ = 0, n_ = 0;
  DevBuf<unsigned long long> mumax_; // two slots: this stage's and the next one's
  unsigned stage_count_ = 0;
  DevBuf<uint8_t> act_a_, act_b_; // per tile: visit in this / the next stage
  uint8_t *act_cur_ = nullptr, *act_next_ = nullptr;
  DevBuf<TileWork> sel_;
  DevBuf<int> nsel_;
  int NN_ = 0;
  std::vector<int32_t> obs_steps_;
  int n_points_ = 0;
  std::vector<double> times_;
  DevBuf<int64_t> idx_;
  DevBuf<double> tgt_, resid_, Jd_, y_, lam_, mu_, lamY_, ls_a_, ls_b_, grad_d_, Ystore_, Sstore_;
  DevBuf<double> Ystore2_, Sstore2_, bclock_;
  double *ystore_[2] = {nullptr, nullptr};
  double *sstore_[2] = {nullptr, nullptr};
  // face points' powder history (three states with faces): NFP_ values per
  // phase state, their stores, checkpoints and adjoint buffers
  size_t NFP_ = 0;
  bool gen_ = false; // the kernel variant with rotation, faces and cube sources
  DevBuf<double> Fstore_, Fstore2_, ck_face_, init_face_, fin_face_, lsf_a_, lsf_b_;
  double *fstore_[2] = {nullptr, nullptr};
  int rec_buf_ = 0;
  DevBuf<MemberData> bmd_;
  DevBuf<BeamState> bbeam_;
  cudaStream_t bst_ = nullptr;
  cudaEvent_t ev_start_ = nullptr, ev_rec_[2] = {nullptr, nullptr}, ev_bwd_[2] = {nullptr, nullptr};
  DevBuf<double> ck_y_, ck_cell_, ck_q_, init_cell_, init_q_, fin_cell_, fin_q_;
  DevBuf<uint8_t> ck_mode_, init_mode_, fin_mode_;
};

} // namespace adm

extern "C" {

int adm_adjoint_create(adm_thermal *h, adm_adjoint **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && out, "null argument");
    *out = nullptr;
    auto *a = new adm::Adjoint(*reinterpret_cast<adm::Thermal *>(h));
    *out = reinterpret_cast<adm_adjoint *>(a);
  });
}

int adm_adjoint_destroy(adm_adjoint *a)
{
  return adm::guard([&] { delete reinterpret_cast<adm::Adjoint *>(a); });
}

int adm_adjoint_set_observations(adm_adjoint *a, int32_t n_obs_steps, int32_t const *obs_steps,
                                 int32_t n_points, int64_t const *node_index, double const *targets)
{
  return adm::guard([&] {
    ADM_REQUIRE(a, "null handle");
    reinterpret_cast<adm::Adjoint *>(a)->set_observations(n_obs_steps, obs_steps, n_points, node_index, targets);
  });
}

int adm_adjoint_objective(adm_adjoint *a, double t0, double dt, int32_t n_steps, double const *y0, double *J,
                          double *y_final)
{
  return adm::guard([&] {
    ADM_REQUIRE(a && y0 && J, "null argument");
    *J = reinterpret_cast<adm::Adjoint *>(a)->objective(t0, dt, n_steps, y0, y_final);
  });
}

int adm_adjoint_gradient(adm_adjoint *a, double t0, double dt, int32_t n_steps, int32_t checkpoint_every,
                         double const *y0, double *J, double *grad, double *y_final)
{
  return adm::guard([&] {
    ADM_REQUIRE(a && y0 && J && grad, "null argument");
    *J = reinterpret_cast<adm::Adjoint *>(a)->gradient(t0, dt, n_steps, checkpoint_every, y0, grad, y_final);
  });
}

int adm_adjoint_checkpoint_interval(adm_adjoint const *a, int32_t *checkpoint_every)
{
  return adm::guard([&] {
    ADM_REQUIRE(a && checkpoint_every, "null argument");
    *checkpoint_every = reinterpret_cast<adm::Adjoint const *>(a)->last_interval();
  });
}

int adm_adjoint_set_flush(adm_adjoint *a, double flush)
{
  return adm::guard([&] {
    ADM_REQUIRE(a, "null handle");
    ADM_REQUIRE(flush >= 0.0 && flush < 1e-3, "flush must be in [0, 1e-3)");
    reinterpret_cast<adm::Adjoint *>(a)->flush_ = flush;
  });
}

int adm_adjoint_vmult_transpose(adm_adjoint *a, double *dst, double const *y, double const *mu, double *grad)
{
  return adm::guard([&] {
    ADM_REQUIRE(a && dst && y && mu, "null argument");
    reinterpret_cast<adm::Adjoint *>(a)->vmult_transpose(dst, y, mu, grad);
  });
}

} // extern "C"
