// MD-platform force bridge (dmffb_md_force_*): the ADMP engine inside an MD engine's own step,
// on the device, in the layout of OpenMM's CUDA platform.
//
// The reference's OpenMM plugin (backend/openmm_dmff_plugin/platforms/cuda/src/
// CudaDMFFKernels.cpp:118-220) copies positions to the host, builds a neighbour list on the
// host (computeNeighborListVoxelHash), runs a TensorFlow graph exported from JAX, keeps the
// induced dipoles on the host for the next step (last_U_ind, :193-195), uploads the forces and
// adds them to the platform's fixed-point force buffer with its addForces kernel
// (kernels/DMFFForce.cu:1-9).  Here every stage stays on the device, on the platform's stream:
//   1. posq (OpenMM's float4 / double4 positions in nm, in the platform's atom order) is gathered
//      into the engine's Angstrom positions through the atom-index array;
//   2. the engine builds its cell-list neighbour list and evaluates energy and forces, the
//      induced-dipole solve starting from the previous step's dipoles, which stay in device
//      memory between steps;
//   3. an epilogue kernel adds the forces, converted to kJ/mol/nm, to the platform's force buffer
//      in its fixed-point format (value * 2^32 as a 64-bit integer, [3][padded atoms]).
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/dmffb200.h"

struct dmffb_md_force {
    dmffb_engine* eng = nullptr;
    int n = 0;
    double* d_pos = nullptr;     // [3n] Angstrom, the system's atom order
    double* d_U = nullptr;       // [3n] induced dipoles (e A), kept across steps
    double* d_forces = nullptr;  // [3n] kJ/mol/A
    dmffb_admp_result last{};
    int lpol = 0;
};

namespace {

__global__ void k_posq_to_pos(int n, const void* posq, int dbl, const int32_t* atom_index, double* pos) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n) return;
    const int a = atom_index ? atom_index[slot] : slot;
    double x, y, z;
    if (dbl) {
        const double4 p = ((const double4*)posq)[slot];
        x = p.x; y = p.y; z = p.z;
    } else {
        const float4 p = ((const float4*)posq)[slot];
        x = p.x; y = p.y; z = p.z;
    }
    pos[3 * a] = x * 10.0;  // nm -> A
    pos[3 * a + 1] = y * 10.0;
    pos[3 * a + 2] = z * 10.0;
}

// forces (kJ/mol/A, system order) -> the platform's fixed-point buffer (kJ/mol/nm * 2^32)
__global__ void k_add_fixed(int n, int padded, const double* forces, const int32_t* atom_index, long long* fb) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n) return;
    const int a = atom_index ? atom_index[slot] : slot;
#pragma unroll
    for (int c = 0; c < 3; ++c) fb[slot + (size_t)c * padded] += (long long)(forces[3 * a + c] * 10.0 * 4294967296.0);
}

}  // namespace

extern "C" {

int dmffb_md_force_create(const dmffb_admp_desc* desc, const double* Q_local, const double* pol, const double* thole,
                          dmffb_md_force** out) {
    if (!desc || !Q_local || !out) return DMFFB_BAD_ARG;
    *out = nullptr;
    dmffb_md_force* f = new dmffb_md_force();
    int st = dmffb_admp_create(desc, &f->eng);
    if (st) {
        if (f->eng) dmffb_destroy(f->eng);
        delete f;
        return st;
    }
    f->n = desc->n_atoms;
    f->lpol = desc->lpol;
    if ((st = dmffb_admp_set_params(f->eng, Q_local, pol, thole))) {
        dmffb_destroy(f->eng);
        delete f;
        return st;
    }
    const size_t b = 3 * (size_t)f->n * sizeof(double);
    if (cudaMalloc((void**)&f->d_pos, b) != cudaSuccess || cudaMalloc((void**)&f->d_U, b) != cudaSuccess ||
        cudaMalloc((void**)&f->d_forces, b) != cudaSuccess || cudaMemset(f->d_U, 0, b) != cudaSuccess) {
        dmffb_md_force_destroy(f);
        return DMFFB_OOM;
    }
    *out = f;
    return DMFFB_OK;
}

int dmffb_md_force_execute(dmffb_md_force* f, const dmffb_md_context* ctx, int32_t include_forces,
                           double* energy_kjmol) {
    if (!f || !ctx || !ctx->posq || (include_forces && !ctx->force_buffer)) return DMFFB_BAD_ARG;
    if (ctx->num_atoms != f->n || ctx->padded_num_atoms < ctx->num_atoms) return DMFFB_BAD_ARG;
    cudaStream_t s = (cudaStream_t)ctx->stream;
    double box[9];
    for (int k = 0; k < 9; ++k) box[k] = ctx->box_nm[k] * 10.0;  // nm -> A
    const unsigned nb = (unsigned)((f->n + 255) / 256);
    k_posq_to_pos<<<nb, 256, 0, s>>>(f->n, ctx->posq, ctx->posq_double, ctx->atom_index, f->d_pos);
    if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
    int st = dmffb_admp_build_neighbors(f->eng, (void*)s, f->d_pos, box);
    if (st) return st;
    st = dmffb_admp_compute(f->eng, (void*)s, f->d_pos, box, nullptr, 0, f->lpol ? f->d_U : nullptr, f->d_forces,
                            &f->last);
    if (st != DMFFB_OK && st != DMFFB_NOT_CONVERGED) return st;
    if (include_forces) {
        k_add_fixed<<<nb, 256, 0, s>>>(f->n, ctx->padded_num_atoms, f->d_forces, ctx->atom_index, ctx->force_buffer);
        if (cudaGetLastError() != cudaSuccess) return DMFFB_CUDA_ERROR;
    }
    if (energy_kjmol) *energy_kjmol = f->last.energy;
    return st;
}

int dmffb_md_force_last_result(const dmffb_md_force* f, dmffb_admp_result* out) {
    if (!f || !out) return DMFFB_BAD_ARG;
    *out = f->last;
    return DMFFB_OK;
}

int dmffb_md_force_dipoles(dmffb_md_force* f, void* stream, double* U_out) {
    if (!f || !U_out) return DMFFB_BAD_ARG;
    if (cudaMemcpyAsync(U_out, f->d_U, 3 * (size_t)f->n * sizeof(double), cudaMemcpyDeviceToDevice,
                        (cudaStream_t)stream) != cudaSuccess)
        return DMFFB_CUDA_ERROR;
    return DMFFB_OK;
}

void dmffb_md_force_destroy(dmffb_md_force* f) {
    if (!f) return;
    if (f->d_pos) cudaFree(f->d_pos);
    if (f->d_U) cudaFree(f->d_U);
    if (f->d_forces) cudaFree(f->d_forces);
    if (f->eng) dmffb_destroy(f->eng);
    delete f;
}

}  // extern "C"
