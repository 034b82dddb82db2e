// Material deposition: boxes along the scan path and their activation of
// cells on the device.
//
// Box generation restates deposition_along_scan_path and
// merge_deposition_paths (source/material_deposition.cc:129-324) for
// three-axis scan paths; the per-step window of boxes follows the driver
// (application/adamantine.hh:1134-1199); the cells a window activates are
// found and activated on the device by Thermal::activate_in_boxes.
#include "capi_common.hpp"
#include "../../include/adamantine_b200_deposition.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace adm
{
namespace
{
struct Box
{
  double lo[3], hi[3], time, c, s;
};

double dist3(double const *a, double const *b)
{
  double const dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// Boxes of one scan path: segments are (end_time, power_modifier, x, y, z)
// rows; the first row gives the start point.
void boxes_along_path(double const *seg, int n_seg, double length, double height, double width, double lead_time,
                      std::vector<Box> &out)
{
  if (n_seg <= 0)
    return;
  double const eps = 1.0e-10, eps_time = 1.0e-10;
  double start_time = 0.0;
  double start[3] = {seg[2], seg[3], seg[4]};
  for (int k = 0; k < n_seg; ++k)
  {
    double const *sg = seg + 5 * k;
    double const end[3] = {sg[2], sg[3], sg[4]};
    if (sg[1] > eps)
    {
      double const seg_len = dist3(end, start);
      double center[3] = {start[0], start[1], start[2]};
      double const velocity = seg_len / (sg[0] - start_time);
      double const c = seg_len != 0. ? (end[0] - start[0]) / seg_len : 1.0;
      double const s = seg_len != 0. ? (end[1] - start[1]) / seg_len : 0.0;
      double box_len = length;
      for (;;)
      {
        double const d_center = dist3(center, start);
        double const t_center = velocity != 0. ? d_center / velocity : 0.;
        double const sx = std::abs(c) * box_len + std::abs(s) * width;
        double const sy = std::abs(c) * width + std::abs(s) * box_len;
        Box b;
        b.lo[0] = center[0] - 0.5 * sx;
        b.hi[0] = center[0] + 0.5 * sx;
        b.lo[1] = center[1] - 0.5 * sy;
        b.hi[1] = center[1] + 0.5 * sy;
        b.lo[2] = center[2] - height;
        b.hi[2] = center[2];
        b.time = std::max(start_time + t_center - lead_time, eps_time);
        b.c = c;
        b.s = s;
        out.push_back(b);
        if (d_center + eps > seg_len)
          break;
        double inc = length;
        if (d_center + length > seg_len)
        {
          inc = seg_len - d_center;
          box_len = seg_len - d_center;
        }
        center[0] += c * inc;
        center[1] += s * inc;
      }
    }
    start[0] = end[0];
    start[1] = end[1];
    start[2] = end[2];
    start_time = sg[0];
  }
}
} // namespace

// Deposition boxes of a thermal handle with their per-step activation window.
class Deposition
{
public:
  Deposition(Thermal &t, int64_t n, double const *lo, double const *hi, double const *time, double const *cosv,
             double const *sinv, double deposition_time, double duration)
      : th_(t), deposition_time_(deposition_time), duration_(duration)
  {
    if (n < 0 || (n > 0 && (!lo || !hi || !time || !cosv || !sinv)))
      throw Error(ADM_ERR_INVALID, "invalid deposition boxes");
    if (n > (int64_t)1 << 31)
      throw Error(ADM_ERR_INVALID, "too many deposition boxes");
    for (int64_t b = 0; b < n; ++b)
    {
      for (int d = 0; d < 3; ++d)
        if (!std::isfinite(lo[3 * b + d]) || !std::isfinite(hi[3 * b + d]))
          throw Error(ADM_ERR_INVALID, "deposition boxes must be finite");
      if (b > 0 && time[b] < time[b - 1])
        throw Error(ADM_ERR_INVALID, "deposition times must be sorted");
    }
    times_.assign(time, time + n);
    ADM_CK(cudaSetDevice(t.device()));
    lo_.alloc(std::max<int64_t>(1, 3 * n));
    hi_.alloc(std::max<int64_t>(1, 3 * n));
    cos_.alloc(std::max<int64_t>(1, n));
    sin_.alloc(std::max<int64_t>(1, n));
    if (n > 0)
    {
      ADM_CK(cudaMemcpy(lo_.p, lo, 3 * n * sizeof(double), cudaMemcpyHostToDevice));
      ADM_CK(cudaMemcpy(hi_.p, hi, 3 * n * sizeof(double), cudaMemcpyHostToDevice));
      ADM_CK(cudaMemcpy(cos_.p, cosv, n * sizeof(double), cudaMemcpyHostToDevice));
      ADM_CK(cudaMemcpy(sin_.p, sinv, n * sizeof(double), cudaMemcpyHostToDevice));
    }
    boxes_.n = n;
    boxes_.lo = lo_.p;
    boxes_.hi = hi_.p;
    boxes_.cosv = cos_.p;
    boxes_.sinv = sin_.p;
    boxes_.cos_host.assign(cosv, cosv + n);
    boxes_.sin_host.assign(sinv, sinv + n);
  }

  int64_t activate_range(int64_t b0, int64_t b1, double new_temperature, double *solution)
  {
    return th_.activate_in_boxes(boxes_, b0, b1, new_temperature, solution);
  }

  // The driver's rule: when the time reaches the end of the last window,
  // the boxes deposited in [time - tol, min(time + max(deposition_time,
  // time_step), duration)) are activated.
  int64_t step(double time, double time_step, double new_temperature, double *solution)
  {
    double const tol = time_step * 1e-6;
    if (!(time - window_end_ > -tol))
      return 0;
    int64_t const start = std::lower_bound(times_.begin(), times_.end(), time - tol) - times_.begin();
    window_end_ = std::min(time + std::max(deposition_time_, time_step), duration_);
    int64_t const end = std::lower_bound(times_.begin(), times_.end(), window_end_) - times_.begin();
    if (start >= end)
      return 0;
    return activate_range(start, end, new_temperature, solution);
  }

private:
  Thermal &th_;
  double deposition_time_, duration_;
  double window_end_ = -1.0;
  std::vector<double> times_;
  DevBuf<double> lo_, hi_, cos_, sin_;
  DeviceBoxes boxes_;
};

} // namespace adm

extern "C" {

int adm_deposition_boxes(adm_source const *sources, int32_t n_sources, double length, double height, double width,
                         double lead_time, int64_t capacity, double *lo, double *hi, double *time, double *cosv,
                         double *sinv, int64_t *n_boxes)
{
  return adm::guard([&] {
    ADM_REQUIRE(n_boxes && (n_sources == 0 || sources), "null argument");
    ADM_REQUIRE(n_sources >= 0 && capacity >= 0, "negative count");
    std::vector<adm::Box> all;
    for (int i = 0; i < n_sources; ++i)
    {
      adm_source const &s = sources[i];
      if (s.type == 2 || s.n_segments <= 0)
        continue;
      ADM_REQUIRE(s.segments, "scan path segments missing");
      adm::boxes_along_path(s.segments, s.n_segments, length, height, width, lead_time, all);
    }
    // merge_deposition_paths: chronological order (ties keep path order)
    std::vector<size_t> perm(all.size());
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return all[a].time < all[b].time; });
    *n_boxes = (int64_t)all.size();
    if (capacity == 0)
      return;
    ADM_REQUIRE(capacity >= (int64_t)all.size(), "capacity smaller than the number of boxes");
    ADM_REQUIRE(lo && hi && time && cosv && sinv, "null output array");
    for (size_t k = 0; k < perm.size(); ++k)
    {
      adm::Box const &b = all[perm[k]];
      for (int d = 0; d < 3; ++d)
      {
        lo[3 * k + d] = b.lo[d];
        hi[3 * k + d] = b.hi[d];
      }
      time[k] = b.time;
      cosv[k] = b.c;
      sinv[k] = b.s;
    }
  });
}

int adm_deposition_create(adm_thermal *h, int64_t n_boxes, double const *lo, double const *hi, double const *time,
                          double const *cosv, double const *sinv, double deposition_time, double duration,
                          adm_deposition **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && out, "null argument");
    *out = nullptr;
    auto *d = new adm::Deposition(*reinterpret_cast<adm::Thermal *>(h), n_boxes, lo, hi, time, cosv, sinv,
                                  deposition_time, duration);
    *out = reinterpret_cast<adm_deposition *>(d);
  });
}

int adm_deposition_destroy(adm_deposition *d)
{
  return adm::guard([&] { delete reinterpret_cast<adm::Deposition *>(d); });
}

int adm_deposition_activate_range(adm_deposition *d, int64_t b0, int64_t b1, double new_temperature,
                                  double *solution, int64_t *n_activated)
{
  return adm::guard([&] {
    ADM_REQUIRE(d && solution, "null argument");
    int64_t const n = reinterpret_cast<adm::Deposition *>(d)->activate_range(b0, b1, new_temperature, solution);
    if (n_activated)
      *n_activated = n;
  });
}

int adm_deposition_step(adm_deposition *d, double time, double time_step, double new_temperature,
                        double *solution, int64_t *n_activated)
{
  return adm::guard([&] {
    ADM_REQUIRE(d && solution, "null argument");
    int64_t const n = reinterpret_cast<adm::Deposition *>(d)->step(time, time_step, new_temperature, solution);
    if (n_activated)
      *n_activated = n;
  });
}

} // extern "C"
