// Stand-alone lattice operators: the drop-ins for TensorLBM's single-purpose
// functions (equilibrium, macroscopic, bounce-back, the boundary planes,
// forces, mass correction, masks and link lists).  The fused step does all of
// this in one pass; these exist so each reference function keeps a one-to-one
// replacement that operates on the caller's buffers.
#include "ops.cuh"
#include "tlbm_bc.cuh"

namespace tlbm {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n, int per_block = kThreads) {
  long long b = (n + per_block - 1) / per_block;
  return (int)(b < 1 ? 1 : (b > 0x7fffffffLL ? 0x7fffffffLL : b));
}

inline int launch_status() { return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH; }

// ---- equilibrium / macroscopic -------------------------------------------

template <class L, typename T>
__global__ void k_equilibrium(long long n, const T* rho, const T* ux, const T* uy, const T* uz, T* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T fe[L::Q];
  equilibrium<L>(rho[i], ux[i], uy[i], L::DIM == 3 ? uz[i] : T(0), fe);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) out[(long long)q * n + i] = fe[q];
}

template <class L, typename T>
__global__ void k_macroscopic(long long n, const T* f, T* rho, T* ux, T* uy, T* uz) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = f[(long long)q * n + i];
  T r, a, b, c;
  macroscopic<L>(v, r, a, b, c);
  rho[i] = r;
  ux[i] = a;
  uy[i] = b;
  if (L::DIM == 3 && uz) uz[i] = c;
}

// ---- bounce-back -----------------------------------------------------------

template <class L, typename T>
__global__ void k_bounce_back(long long n, const T* fin, const uint8_t* mask, T* fout) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool m = mask[i] != 0;
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = fin[(long long)q * n + i];
  if (m) bounce_back<L>(v);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fout[(long long)q * n + i] = v[q];
}

template <class L, typename T>
__global__ void k_moving_wall(long long n, const T* fin, const uint8_t* mask, const T* uw, T* fout) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = fin[(long long)q * n + i];
  if (mask[i]) moving_wall_bounce_back<L>(v, uw[i], uw[n + i], L::DIM == 3 ? uw[2 * n + i] : T(0));
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fout[(long long)q * n + i] = v[q];
}

// ---- boundary planes (in place) -------------------------------------------

template <class L, typename T>
__global__ void k_zou_he_inlet(int nx, int ny, int nz, T* f, BcParams<T> bp, const T* uxp, const T* uyp) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // (z, y) plane index
  if (j >= (long long)ny * nz) return;
  const long long n = (long long)nx * ny * nz;
  const long long cell = j * nx;  // x = 0
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = f[(long long)q * n + cell];
  if constexpr (L::Q == 9) {
    const int y = (int)j;
    const T u = uxp ? uxp[y] : bp.u_in;
    const T uy = uyp ? uyp[y] : bp.uy_in;
    zou_he_inlet_d2q9(v, u, uy);
  } else {
    zou_he_inlet_3d<L>(v, bp.u_in, bp.uy_in, bp.uz_in, bp.one_minus_u);
  }
#pragma unroll
  for (int q = 0; q < L::Q; ++q)
    if (L::cx(q) > 0) f[(long long)q * n + cell] = v[q];
}

template <class L, typename T>
__global__ void k_zou_he_outlet(int nx, int ny, int nz, T* f, BcParams<T> bp) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (long long)ny * nz) return;
  const long long n = (long long)nx * ny * nz;
  const long long cell = j * nx + (nx - 1);
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = f[(long long)q * n + cell];
  if constexpr (L::Q == 9) zou_he_outlet_d2q9(v, bp.rho_out, bp.two_thirds_rho_out, bp.sixth_rho_out);
  else zou_he_outlet_3d<L>(v, bp.rho_out);
#pragma unroll
  for (int q = 0; q < L::Q; ++q)
    if (L::cx(q) < 0) f[(long long)q * n + cell] = v[q];
}

// Free-stream far field, one thread per (y, z) row: a lateral row (y = 0,
// ny-1; with zf also z = 0, nz-1) takes feq(1, u) everywhere; any other row
// takes it at x = 0 and copies x = nx-2 to x = nx-1 (zero gradient).  Lateral
// rows win on the outlet edges, as in boundaries3d.py:515-538.
template <class L, typename T>
__global__ void k_far_field(int nx, int ny, int nz, T* f, T ux, T uy, T uz, bool zf) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // (z, y) index
  if (j >= (long long)ny * nz) return;
  const long long n = (long long)nx * ny * nz;
  const int y = (int)(j % ny);
  const int z = (int)(j / ny);
  const long long row = j * nx;
  T v[L::Q];
  far_field_feq<L>(v, ux, uy, uz);
  const bool lateral = y == 0 || y == ny - 1 || (zf && (z == 0 || z == nz - 1));
  if (lateral) {
    for (int x = 0; x < nx; ++x) {
#pragma unroll
      for (int q = 0; q < L::Q; ++q) f[(long long)q * n + row + x] = v[q];
    }
  } else {
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
      f[(long long)q * n + row] = v[q];
      f[(long long)q * n + row + nx - 1] = f[(long long)q * n + row + nx - 2];
    }
  }
}

template <class L, typename T>
__global__ void k_moving_lid(int nx, int ny, int nz, T* f, T u_lid) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // (z, x) index
  if (j >= (long long)nx * nz) return;
  const long long n = (long long)nx * ny * nz;
  const int x = (int)(j % nx);
  const long long z = j / nx;
  const long long cell = z * nx * ny + (long long)(ny - 1) * nx + x;
  T v[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) v[q] = f[(long long)q * n + cell];
  if constexpr (L::Q == 9) moving_lid_d2q9(v, u_lid);
  else moving_lid_d3q19(v, u_lid);
#pragma unroll
  for (int q = 0; q < L::Q; ++q)
    if (L::cy(q) < 0) f[(long long)q * n + cell] = v[q];
}

// ---- reductions ------------------------------------------------------------

template <int K>
__device__ __forceinline__ void block_reduce_add(double (&v)[K], double* out) {
  __shared__ double sh[K][kThreads / 32];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[k][wid] = v[k];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = lane < kThreads / 32 ? sh[k][lane] : 0.0;
      t = warp_sum(t);
      if (lane == 0) atomicAdd(out + k, t);
    }
  }
}

template <class L, typename T>
__global__ void k_obstacle_force(long long n, const T* f, const uint8_t* mask, double* out) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (!mask[i]) continue;
    T v[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) v[q] = f[(long long)q * n + i];
    T mx, my, mz;
    cell_momentum<L>(v, mx, my, mz);
    acc[0] += 2.0 * double(mx);
    acc[1] += 2.0 * double(my);
    acc[2] += 2.0 * double(mz);
  }
  block_reduce_add<3>(acc, out);
}

template <class L, typename S>
__global__ void k_moment_sums(long long n, const S* f, double* out) {
  using T = typename Storage<S>::T;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
      const double v = double(Storage<S>::load(f[(long long)q * n + i], weight<L, T>(q)));
      r += v;
      jx += L::cx(q) * v;
      jy += L::cy(q) * v;
      jz += L::cz(q) * v;
    }
    acc[0] += r;
    acc[1] += jx;
    acc[2] += jy;
    acc[3] += jz;
  }
  block_reduce_add<4>(acc, out);
}

template <typename T>
__global__ void k_sum(long long count, const T* f, double* out) {
  double acc[1] = {0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
    acc[0] += double(f[i]);
  block_reduce_add<1>(acc, out);
}

// correct_mass: the scale is formed on the device from the float64 sum, so no
// host round trip is needed; torch computes target/current in the field dtype.
template <typename T>
__global__ void k_scale_to_mass(long long count, const T* fin, T* fout, double target, const double* current) {
  const double cur = *current;
  const T cur_t = T(cur);
  const bool skip = fabs(double(cur_t)) < 1e-30;
  const T s = skip ? T(1) : T(target) / cur_t;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
    fout[i] = skip ? fin[i] : fin[i] * s;
}

// ---- masks, flags, links ----------------------------------------------------

// (x - cx)^2 + (y - cy)^2 + (z - cz)^2 <= r^2 in float32 with torch's
// evaluation order and rounding (no fused multiply-add).
__global__ void k_sphere_mask(int nx, int ny, int nz, float cx, float cy, float cz, float r2, uint8_t* out) {
  const long long n = (long long)nx * ny * nz;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = (int)(i % nx);
  const int y = (int)((i / nx) % ny);
  const int z = (int)(i / ((long long)nx * ny));
  const float dx = __fsub_rn((float)x, cx), dy = __fsub_rn((float)y, cy), dz = __fsub_rn((float)z, cz);
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  out[i] = s <= r2 ? 1 : 0;
}

__global__ void k_cylinder_mask(int nx, int ny, float cx, float cy, float r2, uint8_t* out) {
  const long long n = (long long)nx * ny;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = (int)(i % nx);
  const int y = (int)(i / nx);
  const float dx = __fsub_rn((float)x, cx), dy = __fsub_rn((float)y, cy);
  const float s = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  out[i] = s <= r2 ? 1 : 0;
}

__global__ void k_build_flags(long long n, const uint8_t* wall, const uint8_t* obstacle, uint32_t wall_flag,
                              uint8_t* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool w = wall && wall[i];
  const bool o = obstacle && obstacle[i];
  uint32_t v;
  if (wall_flag == TLBM_FLAG_HALFWAY)
    v = (w ? TLBM_FLAG_HALFWAY : 0u) | (o ? (TLBM_FLAG_SOLID | TLBM_FLAG_OBSTACLE) : 0u);
  else
    v = ((w != o) ? TLBM_FLAG_SOLID : 0u) | (o ? TLBM_FLAG_OBSTACLE : 0u);
  flags[i] = (uint8_t)v;
}

// boundary_registry.py:488-575: a population is missing when its pull source
// is solid or lies beyond a non-periodic face
template <class L>
__global__ void k_missing_mask(int nx, int ny, int nz, const uint8_t* solid, int periodic, uint8_t* out) {
  const long long n = (long long)nx * ny * nz;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = (int)(i % nx);
  const int y = (int)((i / nx) % ny);
  const int z = (int)(i / ((long long)nx * ny));
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    int sx = x - L::cx(q), sy = y - L::cy(q), sz = z - L::cz(q);
    bool blocked = false;
    if (sx < 0 || sx >= nx) { if (periodic & 1) sx = (sx + nx) % nx; else blocked = true; }
    if (sy < 0 || sy >= ny) { if (periodic & 2) sy = (sy + ny) % ny; else blocked = true; }
    if (sz < 0 || sz >= nz) { if (periodic & 4) sz = (sz + nz) % nz; else blocked = true; }
    if (!blocked && solid) blocked = solid[((long long)sz * ny + sy) * nx + sx] != 0;
    out[(long long)q * n + i] = blocked ? 1 : 0;
  }
}

constexpr int kLinkChunk = 1024;  // mask bytes per block (256 threads x 4)

__global__ void k_link_count(const uint8_t* mask, long long count, long long* block_counts) {
  const long long base = (long long)blockIdx.x * kLinkChunk;
  int c = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long i = base + k * kThreads + threadIdx.x;
    if (i < count && mask[i]) ++c;
  }
  __shared__ int sh[kThreads / 32];
  int w = c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int k = 0; k < kThreads / 32; ++k) t += sh[k];
    block_counts[blockIdx.x] = t;
  }
}

// exclusive scan of block_counts in place (one block, sequential over tiles)
__global__ void k_link_scan(long long* block_counts, long long nblocks, long long* total) {
  __shared__ long long sh[kThreads];
  long long carry = 0;
  for (long long base = 0; base < nblocks; base += kThreads) {
    const long long i = base + threadIdx.x;
    const long long v = i < nblocks ? block_counts[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
      const long long t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) block_counts[i] = carry + sh[threadIdx.x] - v;
    carry += sh[kThreads - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_link_list(const uint8_t* mask, long long count, const long long* offsets, long long* out) {
  __shared__ int sh[kThreads];
  const long long base = (long long)blockIdx.x * kLinkChunk + (long long)threadIdx.x * 4;
  int c = 0;
  bool hit[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long i = base + k;
    hit[k] = (i < count) && mask[i];
    c += hit[k];
  }
  sh[threadIdx.x] = c;
  __syncthreads();
  for (int o = 1; o < kThreads; o <<= 1) {
    const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  long long pos = offsets[blockIdx.x] + sh[threadIdx.x] - c;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (hit[k]) out[pos++] = base + k;
}

template <class L, typename T>
int run_force(long long n, const T* f, const uint8_t* mask, double* out, cudaStream_t s) {
  if (cudaMemsetAsync(out, 0, 3 * sizeof(double), s) != cudaSuccess) return TLBM_ERR_LAUNCH;
  int blocks = blocks_for(n);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_obstacle_force<L, T><<<blocks, kThreads, 0, s>>>(n, f, mask, out);
  return launch_status();
}

}  // namespace

// ----------------------------------------------------------------------------
// typed runners called from capi.cu
// ----------------------------------------------------------------------------
template <class L, typename T>
int op_equilibrium(long long n, const void* rho, const void* ux, const void* uy, const void* uz, void* out, cudaStream_t s) {
  k_equilibrium<L, T><<<blocks_for(n), kThreads, 0, s>>>(n, (const T*)rho, (const T*)ux, (const T*)uy, (const T*)uz, (T*)out);
  return launch_status();
}
template <class L, typename T>
int op_macroscopic(long long n, const void* f, void* rho, void* ux, void* uy, void* uz, cudaStream_t s) {
  k_macroscopic<L, T><<<blocks_for(n), kThreads, 0, s>>>(n, (const T*)f, (T*)rho, (T*)ux, (T*)uy, (T*)uz);
  return launch_status();
}
template <class L, typename T>
int op_bounce_back(long long n, const void* fin, const uint8_t* mask, void* fout, cudaStream_t s) {
  k_bounce_back<L, T><<<blocks_for(n), kThreads, 0, s>>>(n, (const T*)fin, mask, (T*)fout);
  return launch_status();
}
template <class L, typename T>
int op_moving_wall(long long n, const void* fin, const uint8_t* mask, const void* uw, void* fout, cudaStream_t s) {
  k_moving_wall<L, T><<<blocks_for(n), kThreads, 0, s>>>(n, (const T*)fin, mask, (const T*)uw, (T*)fout);
  return launch_status();
}
template <class L, typename T>
int op_zou_he_inlet(int nx, int ny, int nz, void* f, double u, double uy, double uz, const void* uxp, const void* uyp, cudaStream_t s) {
  const BcParams<T> bp = make_bc_params<T>(u, uy, uz, 1.0, 0.0);
  k_zou_he_inlet<L, T><<<blocks_for((long long)ny * nz), kThreads, 0, s>>>(nx, ny, nz, (T*)f, bp, (const T*)uxp, (const T*)uyp);
  return launch_status();
}
template <class L, typename T>
int op_zou_he_outlet(int nx, int ny, int nz, void* f, double rho_out, cudaStream_t s) {
  const BcParams<T> bp = make_bc_params<T>(0.0, 0.0, 0.0, rho_out, 0.0);
  k_zou_he_outlet<L, T><<<blocks_for((long long)ny * nz), kThreads, 0, s>>>(nx, ny, nz, (T*)f, bp);
  return launch_status();
}
template <class L, typename T>
int op_far_field(int nx, int ny, int nz, void* f, double ux, double uy, double uz, bool z_faces, cudaStream_t s) {
  k_far_field<L, T><<<blocks_for((long long)ny * nz), kThreads, 0, s>>>(nx, ny, nz, (T*)f, T(ux), T(uy), T(uz),
                                                                        z_faces);
  return launch_status();
}
template <class L, typename T>
int op_moving_lid(int nx, int ny, int nz, void* f, double u_lid, cudaStream_t s) {
  k_moving_lid<L, T><<<blocks_for((long long)nx * nz), kThreads, 0, s>>>(nx, ny, nz, (T*)f, T(u_lid));
  return launch_status();
}
template <class L, typename T>
int op_obstacle_force(long long n, const void* f, const uint8_t* mask, double* out, cudaStream_t s) {
  return run_force<L, T>(n, (const T*)f, mask, out, s);
}
template <class L, typename S>
int op_moment_sums(long long n, const void* f, double* out, cudaStream_t s) {
  if (cudaMemsetAsync(out, 0, 4 * sizeof(double), s) != cudaSuccess) return TLBM_ERR_LAUNCH;
  int blocks = blocks_for(n);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_moment_sums<L, S><<<blocks, kThreads, 0, s>>>(n, (const S*)f, out);
  return launch_status();
}
template <typename T>
int op_correct_mass(long long count, const void* fin, void* fout, double target, double* scratch, cudaStream_t s) {
  if (cudaMemsetAsync(scratch, 0, sizeof(double), s) != cudaSuccess) return TLBM_ERR_LAUNCH;
  int blocks = blocks_for(count);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_sum<T><<<blocks, kThreads, 0, s>>>(count, (const T*)fin, scratch);
  if (cudaGetLastError() != cudaSuccess) return TLBM_ERR_LAUNCH;
  k_scale_to_mass<T><<<blocks, kThreads, 0, s>>>(count, (const T*)fin, (T*)fout, target, scratch);
  return launch_status();
}

int op_sphere_mask(int nx, int ny, int nz, double cx, double cy, double cz, double r, uint8_t* out, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  k_sphere_mask<<<blocks_for(n), kThreads, 0, s>>>(nx, ny, nz, (float)cx, (float)cy, (float)cz, (float)(r * r), out);
  return launch_status();
}
int op_cylinder_mask(int nx, int ny, double cx, double cy, double r, uint8_t* out, cudaStream_t s) {
  const long long n = (long long)nx * ny;
  k_cylinder_mask<<<blocks_for(n), kThreads, 0, s>>>(nx, ny, (float)cx, (float)cy, (float)(r * r), out);
  return launch_status();
}
int op_build_flags(long long n, const uint8_t* wall, const uint8_t* obstacle, uint32_t wall_flag, uint8_t* flags,
                   cudaStream_t s) {
  k_build_flags<<<blocks_for(n), kThreads, 0, s>>>(n, wall, obstacle, wall_flag, flags);
  return launch_status();
}
template <class L>
int op_missing_mask(int nx, int ny, int nz, const uint8_t* solid, int periodic, uint8_t* out, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  k_missing_mask<L><<<blocks_for(n), kThreads, 0, s>>>(nx, ny, nz, solid, periodic, out);
  return launch_status();
}
long long op_link_blocks(long long count) { return (count + kLinkChunk - 1) / kLinkChunk; }
int op_link_count(const uint8_t* mask, long long count, long long* block_counts, long long* total, cudaStream_t s) {
  const long long nb = op_link_blocks(count);
  if (nb > 0x7fffffffLL) return TLBM_ERR_SHAPE;
  if (nb == 0) return cudaMemsetAsync(total, 0, sizeof(long long), s) == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
  k_link_count<<<(int)nb, kThreads, 0, s>>>(mask, count, block_counts);
  if (cudaGetLastError() != cudaSuccess) return TLBM_ERR_LAUNCH;
  k_link_scan<<<1, kThreads, 0, s>>>(block_counts, nb, total);
  return launch_status();
}
int op_link_list(const uint8_t* mask, long long count, const long long* offsets, long long* out, cudaStream_t s) {
  const long long nb = op_link_blocks(count);
  if (nb == 0) return TLBM_OK;
  k_link_list<<<(int)nb, kThreads, 0, s>>>(mask, count, offsets, out);
  return launch_status();
}

// explicit instantiations
#define TLBM_INST_LT(L, T)                                                                                   \
  template int op_equilibrium<L, T>(long long, const void*, const void*, const void*, const void*, void*,   \
                                    cudaStream_t);                                                          \
  template int op_macroscopic<L, T>(long long, const void*, void*, void*, void*, void*, cudaStream_t);       \
  template int op_bounce_back<L, T>(long long, const void*, const uint8_t*, void*, cudaStream_t);            \
  template int op_zou_he_inlet<L, T>(int, int, int, void*, double, double, double, const void*, const void*, \
                                     cudaStream_t);                                                         \
  template int op_zou_he_outlet<L, T>(int, int, int, void*, double, cudaStream_t);                          \
  template int op_obstacle_force<L, T>(long long, const void*, const uint8_t*, double*, cudaStream_t);

TLBM_INST_LT(D2Q9, float)
TLBM_INST_LT(D2Q9, double)
TLBM_INST_LT(D3Q19, float)
TLBM_INST_LT(D3Q19, double)
TLBM_INST_LT(D3Q27, float)
TLBM_INST_LT(D3Q27, double)
template int op_moving_wall<D2Q9, float>(long long, const void*, const uint8_t*, const void*, void*, cudaStream_t);
template int op_moving_wall<D2Q9, double>(long long, const void*, const uint8_t*, const void*, void*, cudaStream_t);
template int op_moving_wall<D3Q19, float>(long long, const void*, const uint8_t*, const void*, void*, cudaStream_t);
template int op_moving_wall<D3Q19, double>(long long, const void*, const uint8_t*, const void*, void*, cudaStream_t);
template int op_far_field<D2Q9, float>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_far_field<D2Q9, double>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_far_field<D3Q19, float>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_far_field<D3Q19, double>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_far_field<D3Q27, float>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_far_field<D3Q27, double>(int, int, int, void*, double, double, double, bool, cudaStream_t);
template int op_moving_lid<D2Q9, float>(int, int, int, void*, double, cudaStream_t);
template int op_moving_lid<D2Q9, double>(int, int, int, void*, double, cudaStream_t);
template int op_moving_lid<D3Q19, float>(int, int, int, void*, double, cudaStream_t);
template int op_moving_lid<D3Q19, double>(int, int, int, void*, double, cudaStream_t);
#define TLBM_INST_SUMS(L)                                                                   \
  template int op_moment_sums<L, float>(long long, const void*, double*, cudaStream_t);     \
  template int op_moment_sums<L, double>(long long, const void*, double*, cudaStream_t);    \
  template int op_moment_sums<L, __half>(long long, const void*, double*, cudaStream_t);    \
  template int op_moment_sums<L, __nv_bfloat16>(long long, const void*, double*, cudaStream_t);
TLBM_INST_SUMS(D2Q9)
TLBM_INST_SUMS(D3Q19)
TLBM_INST_SUMS(D3Q27)
template int op_correct_mass<float>(long long, const void*, void*, double, double*, cudaStream_t);
template int op_correct_mass<double>(long long, const void*, void*, double, double*, cudaStream_t);
template int op_missing_mask<D2Q9>(int, int, int, const uint8_t*, int, uint8_t*, cudaStream_t);
template int op_missing_mask<D3Q19>(int, int, int, const uint8_t*, int, uint8_t*, cudaStream_t);
template int op_missing_mask<D3Q27>(int, int, int, const uint8_t*, int, uint8_t*, cudaStream_t);

}  // namespace tlbm
