// Declarations of the stand-alone operator runners (ops.cu).
#pragma once

#include "tlbm_common.cuh"

namespace tlbm {

template <class L, typename T>
int op_equilibrium(long long n, const void* rho, const void* ux, const void* uy, const void* uz, void* out, cudaStream_t s);
template <class L, typename T>
int op_macroscopic(long long n, const void* f, void* rho, void* ux, void* uy, void* uz, cudaStream_t s);
template <class L, typename T>
int op_bounce_back(long long n, const void* fin, const uint8_t* mask, void* fout, cudaStream_t s);
template <class L, typename T>
int op_moving_wall(long long n, const void* fin, const uint8_t* mask, const void* uw, void* fout, cudaStream_t s);
template <class L, typename T>
int op_zou_he_inlet(int nx, int ny, int nz, void* f, double u, double uy, double uz, const void* uxp, const void* uyp,
                    cudaStream_t s);
template <class L, typename T>
int op_zou_he_outlet(int nx, int ny, int nz, void* f, double rho_out, cudaStream_t s);
template <class L, typename T>
int op_moving_lid(int nx, int ny, int nz, void* f, double u_lid, cudaStream_t s);
template <class L, typename T>
int op_far_field(int nx, int ny, int nz, void* f, double ux, double uy, double uz, bool z_faces, cudaStream_t s);
template <class L, typename T>
int op_obstacle_force(long long n, const void* f, const uint8_t* mask, double* out, cudaStream_t s);
template <class L, typename S>
int op_moment_sums(long long n, const void* f, double* out, cudaStream_t s);
template <typename T>
int op_correct_mass(long long count, const void* fin, void* fout, double target, double* scratch, cudaStream_t s);
int op_sphere_mask(int nx, int ny, int nz, double cx, double cy, double cz, double r, uint8_t* out, cudaStream_t s);
int op_cylinder_mask(int nx, int ny, double cx, double cy, double r, uint8_t* out, cudaStream_t s);
int op_build_flags(long long n, const uint8_t* wall, const uint8_t* obstacle, uint32_t wall_flag, uint8_t* flags,
                   cudaStream_t s);
template <class L>
int op_missing_mask(int nx, int ny, int nz, const uint8_t* solid, int periodic, uint8_t* out, cudaStream_t s);
long long op_link_blocks(long long count);
int op_link_count(const uint8_t* mask, long long count, long long* block_counts, long long* total, cudaStream_t s);
int op_link_list(const uint8_t* mask, long long count, const long long* offsets, long long* out, cudaStream_t s);

}  // namespace tlbm
