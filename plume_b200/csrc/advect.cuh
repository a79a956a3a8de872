// Fused clamped-MacCormack advection (advect.cu): one pass per field group, hat kept in shared memory.
#pragma once

#include "common.cuh"

namespace plume {

// The three velocity components advected by themselves (stepper.py:46-52): u, v, w -> u_next, v_next, w_next.
template <class T>
int launch_mac_velocity(const PlumeGridInfo& info, const T* u, const T* v, const T* w, T* u_next, T* v_next,
                        T* w_next, float dt_over_cell, cudaStream_t st);

// Smoke and temperature advected by (u, v, w) (stepper.py:54-58), their values beyond open faces `*_outside`
// when uses_outside == 1. seg_sums (mac_partial_floats floats) receives the smoke line sums of data, hat and
// next per x segment; line_partials (3 * ceil(ny*nz / 256) doubles) their block totals in the layout
// k_budget_factor reads. With `dissipate`, temperature is stored as ambient + (T - ambient) * heat_keep.
template <class T>
int launch_mac_scalars(const PlumeGridInfo& info, const T* u, const T* v, const T* w, const T* smoke,
                       const T* temperature, T* smoke_next, T* temperature_next, float smoke_outside,
                       float heat_outside, int uses_outside, float* seg_sums, double* line_partials, int dissipate,
                       float heat_keep, float ambient, float dt_over_cell, cudaStream_t st);

// x segments of the scalar march, and the floats its segment line sums need.
int mac_segments_for_scalars(const PlumeGridInfo& info);
long long mac_partial_floats(const PlumeGridInfo& info);

}  // namespace plume
