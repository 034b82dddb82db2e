// The state of heat source b of a member at the stage time
// clock[0] + c * clock[1] (position on the scan path, power modifier and the
// derived constants), written to md.beam_state[b]: ScanPath::value /
// get_power_modifier (source/ScanPath.cc:197-275) and GoldakHeatSource /
// ElectronBeamHeatSource / CubeHeatSource::update_time
// (source/GoldakHeatSource.cc:24-44, source/ElectronBeamHeatSource.cc:24-45,
// source/CubeHeatSource.cc:45-49).
#pragma once

#include "device_types.cuh"

namespace adm
{
__device__ __forceinline__ void prepare_beam(MemberData const &md, int b, double c)
{
  double const t = md.clock[0] + c * md.clock[1];
  BeamDesc const &bd = md.beams[b];
  BeamState st;
  st.type = bd.type;
  st.depth = bd.depth;
  st.radius_squared = bd.radius_squared;
  st.five_r2 = 5. * bd.radius_squared;
  st.inv_r2 = 0.0;
  st.inv_d2 = 0.0;
  st.inv_d = 0.0;
  st.log01 = md.log_01;
  st.alpha = 0.0;
  for (int d = 0; d < 3; ++d)
  {
    st.cube_min[d] = bd.cube_min[d];
    st.cube_max[d] = bd.cube_max[d];
    st.center[d] = 0.0;
  }
  st.cube_value = bd.cube_value;
  if (bd.type == 2)
  {
    st.on = (t > bd.cube_start_time) && (t < bd.cube_end_time);
  }
  else
  {
    int const n = bd.n_segments;
    double const *sg = bd.segments;
    double pmod = 0.0;
    if (n == 0 || t > sg[(n - 1) * 5])
    {
      double const low = -1.7976931348623157e308;
      st.center[0] = st.center[1] = st.center[2] = low;
    }
    else
    {
      // first segment whose end time is >= t (end times are non-decreasing)
      int lo = 0, hi = n - 1;
      while (lo < hi)
      {
        int const mid = (lo + hi) / 2;
        if (t > sg[mid * 5])
          lo = mid + 1;
        else
          hi = mid;
      }
      int const cur = lo;
      double st_t, sp[3];
      if (cur > 0)
      {
        st_t = sg[(cur - 1) * 5];
        for (int d = 0; d < 3; ++d)
          sp[d] = sg[(cur - 1) * 5 + 2 + d];
      }
      else
      {
        st_t = 0.0;
        for (int d = 0; d < 3; ++d)
          sp[d] = sg[cur * 5 + 2 + d];
      }
      double const et = sg[cur * 5];
      for (int d = 0; d < 3; ++d)
        st.center[d] = sp[d] + (sg[cur * 5 + 2 + d] - sp[d]) / (et - st_t) * (t - st_t);
      pmod = sg[cur * 5 + 1];
    }
    st.on = pmod > 0.0;
    if (bd.type == 0)
    {
      st.alpha = 2.0 * bd.absorption_efficiency * bd.max_power * pmod /
                 (bd.radius_squared * bd.depth * md.pi_over_3_to_1p5);
      st.inv_r2 = 1.0 / bd.radius_squared;
      st.inv_d2 = 1.0 / (bd.depth * bd.depth);
    }
    else
    {
      st.alpha = -bd.absorption_efficiency * bd.max_power * pmod * md.log_01 /
                 (3.14159265358979323846 * bd.radius_squared * bd.depth);
      st.inv_d = 1.0 / bd.depth;
      st.inv_r2 = 1.0 / bd.radius_squared;
    }
  }
  md.beam_state[b] = st;
}
} // namespace adm
