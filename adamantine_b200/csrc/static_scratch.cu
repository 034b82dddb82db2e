// adm_vmult_host_static: the host-buffer vmult with its device staging in a
// file-scope static array instead of cudaMalloc'ed vectors.
#include "thermal.hpp"

#include <mutex>
#include <string>

namespace
{
constexpr size_t kMaxNodes = ADM_STATIC_SCRATCH_MAX_NODES;

// src staging at [0, kMaxNodes), dst staging at [kMaxNodes, 2 kMaxNodes).
// 256-byte alignment keeps both halves valid TMA sources.
__device__ __align__(256) double g_static_scratch[2 * kMaxNodes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {};

// Device address of the static array on `device` (looked up once per device,
// with that device current). Host code must not use the symbol itself: on
// the host it names a stand-in, not device memory.
double *scratch_on(int device)
{
  if (device < 0 || device >= kMaxDevices)
    throw adm::Error(ADM_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[device])
  {
    int current = 0;
    ADM_CK(cudaGetDevice(&current));
    ADM_CK(cudaSetDevice(device));
    void *p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&p, g_static_scratch);
    cudaSetDevice(current);
    ADM_CK(e);
    g_scratch_addr[device] = static_cast<double *>(p);
  }
  return g_scratch_addr[device];
}

} // namespace

namespace adm
{
void set_last_error(std::string const &msg);
}

extern "C" int adm_vmult_host_static(adm_thermal *h, double *dst_host, double const *src_host)
{
  try
  {
    if (!h || !dst_host || !src_host)
      throw adm::Error(ADM_ERR_INVALID, "null argument");
    auto *t = reinterpret_cast<adm::Thermal *>(h);
    size_t const n = t->m();
    if (n > kMaxNodes)
      throw adm::Error(ADM_ERR_INVALID,
                       "adm_vmult_host_static: the node vector has " + std::to_string(n) +
                           " entries; the static staging array holds at most " +
                           std::to_string(kMaxNodes) + " (use adm_vmult_host)");
    double *const base = scratch_on(t->device());
    double *const src_d = base;
    double *const dst_d = base + kMaxNodes;
    ADM_CK(cudaSetDevice(t->device()));
    ADM_CK(cudaMemcpyAsync(src_d, src_host, n * sizeof(double), cudaMemcpyHostToDevice, t->stream()));
    t->vmult(dst_d, src_d, false);
    ADM_CK(cudaMemcpyAsync(dst_host, dst_d, n * sizeof(double), cudaMemcpyDeviceToHost, t->stream()));
    t->synchronize();
    return ADM_OK;
  }
  catch (adm::Error const &e)
  {
    adm::set_last_error(e.what());
    return e.code;
  }
  catch (std::exception const &e)
  {
    adm::set_last_error(e.what());
    return ADM_ERR_INVALID;
  }
}
