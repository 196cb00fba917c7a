// Doubly periodic 2D decaying turbulence (vorticity form) in FP32: plan object
// used by the C ABI (tb_turb_*) and by the request server.  Not public.
#pragma once

#include <cuda_runtime.h>

#include "tb_internal.h"

struct tb_turb;

namespace tb {

// q0_spec: initial vorticity coefficients, complex128 interleaved, layout
// (Nx/2+1, Ny) with x fastest (rfft along x, fft along y, unnormalised).
tb_turb* turb_create(tb_context* ctx, const tb_problem_desc& d, const double* q0_spec);
void turb_destroy(tb_turb* T);
// Replace q_n (layout of q0_spec); the step history restarts.
void turb_set(tb_turb* T, const double* q0_spec);
cudaStream_t turb_stream(const tb_turb* T);
// Enqueue steps on the plan's stream (returns without waiting).
void turb_launch_steps(tb_turb* T, double dt, int steps);
// Step graphs for dt, built ahead of the first launch.
void turb_prepare(tb_turb* T, double dt);
size_t turb_device_bytes(const tb_turb* T);
size_t turb_field_doubles(const tb_turb* T);
// Vorticity coefficients to host, complex128 (Nx/2+1, Ny), x fastest (waits).
void turb_fetch(tb_turb* T, double* host);
size_t turb_estimate_bytes(int Nx, int Ny, int timestepper);

}  // namespace tb
