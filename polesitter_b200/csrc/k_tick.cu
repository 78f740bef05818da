// The caller's tick loop on the device: ids reset, then (after prepare and
// calc) the velocity permutation through ids and the semi-implicit Euler
// step.
//
// Reference: the loop every polesitter user writes around ps_calc_forces,
// README.md:65-111 (the same steps in demo/unary.c:117-189):
//   ids[i] = i                                         (README.md:67-70)
//   prepare + calc: x, y, z, mass, ids end sorted, forces in sorted order
//   v_new[i] = v[ids[i]]                               (README.md:82-93)
//   if mass[i] > 0: v += (f / m) * dt; x += v * dt     (README.md:98-110)
// Each step is rounded as the C expression is written (no contraction), so
// the update is bit-identical to the loop compiled with strict IEEE float.
// Bound: HBM, 40 B read (8 of them gathered) + 24 B written per particle.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

__global__ void __launch_bounds__(256) k_tick_reset_ids(uint32_t* __restrict__ id, size_t n) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        id[i] = (uint32_t)i;
}

__global__ void __launch_bounds__(256) k_tick_euler(TickState t, size_t n, float dt) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t old = t.id[i];
        if (old >= n) continue;  // ids are a permutation of 0..n-1 after the reset
        float vx = t.vx_in[old], vy = t.vy_in[old], vz = t.vz_in[old];
        const float m = t.m[i];
        if (m > 0.0f) {
            vx = __fadd_rn(vx, __fmul_rn(__fdiv_rn(t.fx[i], m), dt));
            vy = __fadd_rn(vy, __fmul_rn(__fdiv_rn(t.fy[i], m), dt));
            vz = __fadd_rn(vz, __fmul_rn(__fdiv_rn(t.fz[i], m), dt));
            t.x[i] = __fadd_rn(t.x[i], __fmul_rn(vx, dt));
            t.y[i] = __fadd_rn(t.y[i], __fmul_rn(vy, dt));
            t.z[i] = __fadd_rn(t.z[i], __fmul_rn(vz, dt));
        }
        t.vx_out[i] = vx;
        t.vy_out[i] = vy;
        t.vz_out[i] = vz;
    }
}

void launch_tick_reset_ids(uint32_t* id, size_t n, int grid, cudaStream_t st) {
    k_tick_reset_ids<<<grid, 256, 0, st>>>(id, n);
}

void launch_tick_euler(const TickState& t, size_t n, float dt, int grid, cudaStream_t st) {
    k_tick_euler<<<grid, 256, 0, st>>>(t, n, dt);
}

}  // namespace psg
