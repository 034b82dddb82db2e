// Checkpoint / restart of a thermal handle (ThermalPhysics::save_checkpoint /
// load_checkpoint, source/ThermalPhysics.templates.hh:974-1185).
//
// Flat little-endian file:
//   "ADMCKPT1", int32 version, int32 dim, degree, n_states, n_cells[3],
//   int64 n_nodes, n_cells, int32 n_slots, int32 nf, double time,
//   per cell: uint8 active, uint8 material id, uint8 has_melted,
//             double cos, double sin,
//   double cell state [n_states][n_cells] (the per-point ratios averaged to
//   the cells, as the reference stores them), double solution [n_nodes],
//   then the exact phase history: uint8 powder mode [n_cells],
//   double powder value [n_cells], double per-point powder [n_cells][NN],
//   double liquid sum [n_cells], double face powder [n_slots][6][nf].
// A restart with exact = 0 follows the reference (cell states broadcast to
// the points); exact = 1 restores the per-point history, so the continued
// run is bit-identical to an uninterrupted one.
#include "capi_common.hpp"

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

namespace adm
{
namespace
{
constexpr char kMagic[8] = {'A', 'D', 'M', 'C', 'K', 'P', 'T', '1'};

struct File
{
  std::FILE *f = nullptr;
  File(char const *path, char const *mode) : f(std::fopen(path, mode)) {}
  ~File()
  {
    if (f)
      std::fclose(f);
  }
};

void put(std::FILE *f, void const *p, size_t n)
{
  if (n && std::fwrite(p, 1, n, f) != n)
    throw Error(ADM_ERR_INVALID, "checkpoint write failed");
}
void get(std::FILE *f, void *p, size_t n)
{
  if (n && std::fread(p, 1, n, f) != n)
    throw Error(ADM_ERR_INVALID, "checkpoint file is truncated");
}
template <class T>
std::vector<T> dev_to_host(T const *d, size_t n, cudaStream_t s)
{
  std::vector<T> h(n);
  if (n && d)
    ADM_CK(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  return h;
}
} // namespace

struct Checkpoint
{
  static void save(Thermal &t, char const *path, double time, double const *solution)
  {
    if (!t.setup_done_)
      throw Error(ADM_ERR_INVALID, "setup() has not been called");
    ADM_CK(cudaSetDevice(t.device_));
    cudaStream_t const st = t.stream_;
    size_t const C = t.mesh_.n_cells, N = t.mesh_.n_nodes;
    int const NN = (t.mesh_.deg + 1) * (t.mesh_.deg + 1) * (t.mesh_.deg + 1);
    int const NF = (t.mesh_.deg + 1) * (t.mesh_.deg + 1);
    // the cells' state as the reference saves it
    t.set_state_to_material_properties();
    auto state = dev_to_host(t.state_d_.p, (size_t)t.ns_ * C, st);
    auto sol = dev_to_host(solution, N, st);
    auto hm = dev_to_host(t.has_melted_d_.p, C, st);
    bool const ns3 = t.ns_ == 3;
    auto pmode = ns3 ? dev_to_host(t.powder_mode_.p, C, st) : std::vector<uint8_t>(C, 0);
    auto pcell = ns3 ? dev_to_host(t.powder_cell_.p, C, st) : std::vector<double>(C, 0.0);
    auto pq = ns3 ? dev_to_host(t.powder_q_.p, C * NN, st) : std::vector<double>(C * NN, 0.0);
    auto lsum = t.ns_ > 1 ? dev_to_host(t.liquid_sum_.p, C, st) : std::vector<double>(C, 0.0);
    int const n_slots = (ns3 && !t.adiabatic_only_) ? t.topo_.n_slots : 0;
    auto fp = dev_to_host(t.face_powder_.p, (size_t)n_slots * 6 * NF, st);
    ADM_CK(cudaStreamSynchronize(st));
    File fh(path, "wb");
    if (!fh.f)
      throw Error(ADM_ERR_INVALID, std::string("cannot open checkpoint file for writing: ") + path);
    int32_t const head[9] = {1, 3, t.mesh_.deg, t.ns_, t.mesh_.nc[0], t.mesh_.nc[1], t.mesh_.nc[2], n_slots, NF};
    int64_t const sizes[2] = {(int64_t)N, (int64_t)C};
    put(fh.f, kMagic, 8);
    put(fh.f, head, sizeof(head));
    put(fh.f, sizes, sizeof(sizes));
    put(fh.f, &time, sizeof(time));
    put(fh.f, t.active_.data(), C);
    put(fh.f, t.matid_.data(), C);
    put(fh.f, hm.data(), C);
    put(fh.f, t.cos_.data(), C * sizeof(double));
    put(fh.f, t.sin_.data(), C * sizeof(double));
    put(fh.f, state.data(), state.size() * sizeof(double));
    put(fh.f, sol.data(), N * sizeof(double));
    put(fh.f, pmode.data(), C);
    put(fh.f, pcell.data(), C * sizeof(double));
    put(fh.f, pq.data(), pq.size() * sizeof(double));
    put(fh.f, lsum.data(), C * sizeof(double));
    put(fh.f, fp.data(), fp.size() * sizeof(double));
    if (std::fflush(fh.f) != 0)
      throw Error(ADM_ERR_INVALID, "checkpoint write failed");
  }

  static double load(Thermal &t, char const *path, bool exact, double *solution)
  {
    File fh(path, "rb");
    if (!fh.f)
      throw Error(ADM_ERR_INVALID, std::string("cannot open checkpoint file: ") + path);
    char magic[8];
    get(fh.f, magic, 8);
    if (std::memcmp(magic, kMagic, 8) != 0)
      throw Error(ADM_ERR_INVALID, "not a checkpoint file");
    int32_t head[9];
    int64_t sizes[2];
    double time = 0.0;
    get(fh.f, head, sizeof(head));
    get(fh.f, sizes, sizeof(sizes));
    get(fh.f, &time, sizeof(time));
    size_t const C = t.mesh_.n_cells, N = t.mesh_.n_nodes;
    int const NN = (t.mesh_.deg + 1) * (t.mesh_.deg + 1) * (t.mesh_.deg + 1);
    if (head[0] != 1 || head[1] != 3 || head[2] != t.mesh_.deg || head[3] != t.ns_ || head[4] != t.mesh_.nc[0] ||
        head[5] != t.mesh_.nc[1] || head[6] != t.mesh_.nc[2] || sizes[0] != (int64_t)N || sizes[1] != (int64_t)C)
      throw Error(ADM_ERR_INVALID, "checkpoint does not match the handle's mesh, element or material states");
    int const n_slots = head[7], NF = head[8];
    std::vector<uint8_t> active(C), matid(C), hm(C), pmode(C);
    std::vector<double> cs(C), sn(C), state((size_t)t.ns_ * C), sol(N), pcell(C), pq(C * NN), lsum(C),
        fp((size_t)n_slots * 6 * NF);
    get(fh.f, active.data(), C);
    get(fh.f, matid.data(), C);
    get(fh.f, hm.data(), C);
    get(fh.f, cs.data(), C * sizeof(double));
    get(fh.f, sn.data(), C * sizeof(double));
    get(fh.f, state.data(), state.size() * sizeof(double));
    get(fh.f, sol.data(), N * sizeof(double));
    get(fh.f, pmode.data(), C);
    get(fh.f, pcell.data(), C * sizeof(double));
    get(fh.f, pq.data(), pq.size() * sizeof(double));
    get(fh.f, lsum.data(), C * sizeof(double));
    get(fh.f, fp.data(), fp.size() * sizeof(double));
    ADM_CK(cudaSetDevice(t.device_));
    cudaStream_t const st = t.stream_;
    // load_checkpoint: the cells, then setup_dofs + the inverse mass
    t.set_cells(active.data(), matid.data(), nullptr, cs.data(), sn.data());
    t.setup();
    t.has_melted_ = hm;
    ADM_CK(cudaMemcpyAsync(t.has_melted_d_.p, hm.data(), C, cudaMemcpyHostToDevice, st));
    ADM_CK(cudaMemcpyAsync(t.state_d_.p, state.data(), state.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    ADM_CK(cudaMemcpyAsync(solution, sol.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    if (exact)
    {
      if (t.ns_ == 3)
      {
        ADM_CK(cudaMemcpyAsync(t.powder_mode_.p, pmode.data(), C, cudaMemcpyHostToDevice, st));
        ADM_CK(cudaMemcpyAsync(t.powder_cell_.p, pcell.data(), C * sizeof(double), cudaMemcpyHostToDevice, st));
        ADM_CK(cudaMemcpyAsync(t.powder_q_.p, pq.data(), pq.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        int const cur_slots = !t.adiabatic_only_ ? t.topo_.n_slots : 0;
        if (cur_slots != n_slots)
          throw Error(ADM_ERR_INVALID, "checkpoint face data does not match the boundary of the handle");
        if (n_slots)
          ADM_CK(cudaMemcpyAsync(t.face_powder_.p, fp.data(), fp.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 st));
      }
      if (t.ns_ > 1)
        ADM_CK(cudaMemcpyAsync(t.liquid_sum_.p, lsum.data(), C * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    else
    {
      // MaterialProperty::set_cell_state + get_state_from_material_properties
      t.get_state_from_material_properties();
    }
    ADM_CK(cudaStreamSynchronize(st));
    return time;
  }
};

} // namespace adm

extern "C" {

int adm_save_checkpoint(adm_thermal *h, char const *path, double time, double const *solution)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && path && solution, "null argument");
    adm::Checkpoint::save(*reinterpret_cast<adm::Thermal *>(h), path, time, solution);
  });
}

int adm_load_checkpoint(adm_thermal *h, char const *path, int32_t exact, double *time, double *solution)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && path && solution, "null argument");
    double const t = adm::Checkpoint::load(*reinterpret_cast<adm::Thermal *>(h), path, exact != 0, solution);
    if (time)
      *time = t;
  });
}

} // extern "C"
