// Device-side data of the B200 thermal hot path.
//
// One "member" is one thermal problem (operator + its state); the single
// operator API uses member 0, the batched ensemble uses many. Everything a
// kernel needs about a member lives in MemberData (device memory), so one
// launch can serve a ragged list of (member, tile) work items.
#pragma once

#include <cstdint>

namespace adm
{
constexpr int kMaxMaterials = 4;
constexpr int kNStateProps = 8;
constexpr int kMaxStates = 3;
constexpr int kMaxPoly = 5;
constexpr int kTableSize = 12;
constexpr int kNProps = 5;
constexpr int kMaxBeams = 4;

// StateProperty order of source/types.hh:40-49
enum StateProp
{
  P_DENSITY = 0,
  P_SPECIFIC_HEAT,
  P_KX,
  P_KY,
  P_KZ,
  P_EMISSIVITY,
  P_RAD_COEF,
  P_CONV_COEF
};
// Property order of source/types.hh:88-96
enum Prop
{
  Q_LIQUIDUS = 0,
  Q_SOLIDUS,
  Q_LATENT,
  Q_RAD_TINF,
  Q_CONV_TINF
};
enum BoundaryBits
{
  B_ADIABATIC = 1,
  B_RADIATIVE = 2,
  B_CONVECTIVE = 4
};

// Sticky device error codes (MemberData::error)
enum DeviceError
{
  DERR_NONE = 0,
  DERR_NONFINITE = 1, // non-finite value in a finalized node
  DERR_BAD_WORK = 2,  // malformed work list entry
  DERR_TMA_TIMEOUT = 3 // a brick copy did not arrive within the wait limit
};

// cell_info bits
constexpr uint32_t CI_ACTIVE = 1u;
constexpr int CI_FACE_SHIFT = 1;      // bits 1..6: face is on the active boundary
constexpr int CI_INTERFACE_SHIFT = 8; // bits 8..13: that face borders an inactive cell
constexpr int CI_MAT_SHIFT = 16;      // bits 16..19: material id

struct BeamDesc
{
  int type; // 0 goldak, 1 electron beam, 2 cube
  int n_segments;
  double const *segments; // device, n x 5 (end_time, pmod, x, y, z)
  double depth;
  double absorption_efficiency;
  double radius_squared;
  double max_power;
  double cube_start_time, cube_end_time, cube_value;
  double cube_min[3], cube_max[3];
};

struct MaterialDesc
{
  int n_materials, n_states, use_table, p_order;
  int prop_deg[kNStateProps]; // highest nonzero polynomial coefficient
  int isotropic;              // k_x, k_y, k_z identical everywhere
  int pad;
  double poly[kMaxMaterials][kNStateProps][kMaxStates][kMaxPoly];
  double table[kMaxMaterials][kNStateProps][kMaxStates][kTableSize][2];
  double props[kMaxMaterials][kNProps];
};

// Heat source state at one stage time (written by the stage-prepare kernel).
struct BeamState
{
  int type;
  int on;
  double center[3];
  double alpha;
  double depth, radius_squared, five_r2, inv_r2, inv_d2, inv_d, log01;
  double cube_min[3], cube_max[3], cube_value;
};

// Everything about one member that kernels read or write.
struct MemberData
{
  // node vectors (pitch-padded full grid)
  double *y;    // solution
  double *za;   // stage vector A
  double *zb;   // stage vector B
  double *s;    // RK running sum of dt*b_j*f_j
  double *f0;   // stored first stage derivative (RK3)
  double *acc;  // partial sums of tile-shared nodes
  double const *inv_mass;
  // cells
  uint32_t const *cell_info;
  uint8_t *powder_mode; // 0 uniform zero, 1 uniform value, 2 per-qp values
  double *powder_cell;
  double *powder_q;     // [C][Q]
  double *liquid_sum;   // [C]: sum over the cell's qp of the liquid ratio
  int32_t const *face_slot;
  double *face_powder;  // [slot][6][NF]
  double const *cosv, *sinv;
  uint32_t const *tile_nbr; // 27-bit neighbour-activity mask per tile (bit 13: the tile itself)
  double *halo;             // two-pass schedule: [n_tiles][halo size] partial sums of the
                            // nodes on each tile's upper brick faces
  MaterialDesc const *mat;
  BeamState *beam_state; // [kMaxBeams], current stage
  double *clock;        // [0] stage base time, [1] dt
  int32_t *error;       // sticky error word
  int n_beams;
  int has_rotation;
  BeamDesc beams[kMaxBeams];
  double pi_over_3_to_1p5;
  double log_01;
};

struct TileWork
{
  int32_t member;
  int32_t tile;
  uint32_t xyz; // tile coordinates packed by pack_tile (no division in kernels)
};

// Tile coordinates in one word: x in bits 0-10, y in 11-21, z in 22-31.
__host__ __device__ inline uint32_t pack_tile(int tx, int ty, int tz)
{
  return (uint32_t)tx | ((uint32_t)ty << 11) | ((uint32_t)tz << 22);
}

// Mesh and stage description passed by value to the tile kernel.
struct KernelArgs
{
  TileWork const *work;
  MemberData const *members;
  // explicit vectors for the operator modes (member 0 only)
  double const *vsrc;
  double *vdst;
  double *y_override; // caller-owned solution vector (member 0), or null
  int mode;     // 0 vmult, 1 vmult_add, 2 stage
  int atomic;   // 1: all colours in one launch, node sums by atomics
  int blocked;  // 1: each CTA takes one contiguous run of work items
  int *claim;   // non-null: items after each CTA's first are claimed from this
                // counter (zero at the launch), dynamic load balance
  int cells_per_thread; // FE_Q(1) cell kernel: 1, 2 (stacked in z) or 4 (the column variant) per thread
  int two_pass;         // two-pass schedule: owners write, upper-face partial sums to md.halo
  int tile_pairs;       // atomic FE_Q(2): work items are z-pairs of tiles (128-cell blocks)
  int stage;
  int last;     // last stage of the step (updates y)
  int n_stages; // 1 forward Euler
  int store_f0;
  int src_sel; // stage input: 0 y, 1 za, 2 zb
  int dst_sel; // stage output: 1 za, 2 zb
  int has_f0;
  double c_stage;   // stage time = clock[0] + c_stage * clock[1]
  double a_next;    // coefficient of f_i in the next stage input
  double a_next_f0; // coefficient of the stored f_0 in the next stage input
  double b_i;       // weight of f_i in the update
  // mesh
  int nc[3], nn[3], nt[3];
  int pitch;
  int faces; // !adiabatic_only
  int boundary_type[6];
  int interface_type;
  double h[3], origin[3];
  double vol_over_h2[3]; // cell volume / h_d^2
  double vol_over_h[3];  // cell volume / h_d
  double vol;            // cell volume
  double inv_h[3];       // 1 / h_d
  double S[3][3];        // S[q][i] = phi_i(x_q)
  double D[3][3];        // collocation derivative at the quadrature points
  double G[3][3];        // G = D S: nodal-basis derivative at the quadrature points
  double qw[3];          // 1D quadrature weights on [0,1]
  double qx[3];          // 1D quadrature points on [0,1]
  // per Gauss point q (lexicographic, up to 27): W_q vol / h_x^2,
  // W_q vol / h_y^2, W_q vol / h_z^2, W_q vol, with W_q the product weight
  double cw[27][4];
};

// L2 eviction priority for stores whose lines should outlive a streaming
// read that follows: the zeroed target of the atomic write-out (its FP64
// reductions then find the lines in L2 instead of fetching them from DRAM)
// and the two-pass halo sums (read back by the gather pass).
#ifdef __CUDACC__
__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_keep(double *p, double v, uint64_t pol)
{
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep2(double *p, double v0, double v1, uint64_t pol)
{
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v0), "d"(v1), "l"(pol)
               : "memory");
}
#endif

} // namespace adm
