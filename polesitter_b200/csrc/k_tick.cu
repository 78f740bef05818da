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

// Many systems in one array (the batched ensemble): ids and velocities are
// each system's own, system k at [sys_off[k], sys_off[k + 1]); positions keep
// their system across a tick (each system is sorted within its range).
__global__ void __launch_bounds__(256) k_forest_reset_ids(uint32_t* __restrict__ id, size_t n,
                                                          const uint32_t* __restrict__ part_sys,
                                                          const uint32_t* __restrict__ sys_off) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        id[i] = (uint32_t)(i - sys_off[part_sys[i]]);
}

__global__ void __launch_bounds__(256) k_forest_euler(TickState t, size_t n, float dt,
                                                      const uint32_t* __restrict__ part_sys,
                                                      const uint32_t* __restrict__ sys_off) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t k = part_sys[i];
        const uint32_t lo = sys_off[k], nk = sys_off[k + 1] - lo;
        const uint32_t old = t.id[i];
        if (old >= nk) continue;  // ids are a permutation of 0..nk-1 after the reset
        float vx = t.vx_in[lo + old], vy = t.vy_in[lo + old], vz = t.vz_in[lo + old];
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

// a one-particle system's root is a leaf with no group to sum it: its only
// P2P term is the zero self-interaction (polesitter.h:1279-1449)
__global__ void k_forest_single_forces(const uint32_t* __restrict__ sys_off, uint32_t nsys,
                                       float* __restrict__ fx, float* __restrict__ fy,
                                       float* __restrict__ fz) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nsys;
         k += gridDim.x * blockDim.x) {
        if (sys_off[k + 1] - sys_off[k] == 1u) {
            fx[sys_off[k]] = 0.f;
            fy[sys_off[k]] = 0.f;
            fz[sys_off[k]] = 0.f;
        }
    }
}

void launch_tick_reset_ids(uint32_t* id, size_t n, int grid, cudaStream_t st) {
    k_tick_reset_ids<<<grid, 256, 0, st>>>(id, n);
}

void launch_tick_euler(const TickState& t, size_t n, float dt, int grid, cudaStream_t st) {
    k_tick_euler<<<grid, 256, 0, st>>>(t, n, dt);
}

void launch_forest_reset_ids(uint32_t* id, size_t n, const uint32_t* part_sys,
                             const uint32_t* sys_off, int grid, cudaStream_t st) {
    k_forest_reset_ids<<<grid, 256, 0, st>>>(id, n, part_sys, sys_off);
}

void launch_forest_euler(const TickState& t, size_t n, float dt, const uint32_t* part_sys,
                         const uint32_t* sys_off, int grid, cudaStream_t st) {
    k_forest_euler<<<grid, 256, 0, st>>>(t, n, dt, part_sys, sys_off);
}

void launch_forest_single_forces(const uint32_t* sys_off, uint32_t nsys, float* fx, float* fy,
                                 float* fz, cudaStream_t st) {
    k_forest_single_forces<<<(nsys + 255) / 256, 256, 0, st>>>(sys_off, nsys, fx, fy, fz);
}

}  // namespace psg
