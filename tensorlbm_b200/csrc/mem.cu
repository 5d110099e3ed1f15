// Link-wise momentum-exchange sums behind TensorLBM's MEM drag variants
// (momentum_exchange.py:75-360): for each fluid cell x marked "near" and each
// direction q >= 1 whose periodic neighbour x + c_q is solid (a fluid->solid
// link), the per-link value (f_q(x) + f_opp(q)(x + c_q)) times an optional
// 1 / max(q_wall, 1e-6) weight, summed per direction in FP64, and the number
// of such links per direction.  The standard, Galilean-invariant,
// background-subtracted and BFL-weighted forces are fixed linear
// combinations of these 2Q numbers (formed on the host).
//
// One pass over the near mask (1 byte per cell); the populations and solid
// neighbours are read only for near cells, so the kernel is bound by the
// mask read.  Each warp skips its row segment when no lane is near; otherwise
// per direction a warp sum of the link values and a ballot count go to a
// block accumulator in shared memory, then once per block to global memory.
#include "tlbm_step.cuh"

namespace tlbm {
namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class L, typename S>
__global__ void __launch_bounds__(256) k_link_sums(const S* __restrict__ f, const uint8_t* __restrict__ solid,
                                                   const uint8_t* __restrict__ near, const float* __restrict__ q_wall,
                                                   int q_per_direction, int nx, int ny, int nz,
                                                   double* __restrict__ sums) {
  constexpr int Q = L::Q;
  __shared__ double acc[2 * Q];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < 2 * Q; i += blockDim.x * blockDim.y) acc[i] = 0.0;
  __syncthreads();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const long long n = (long long)nx * ny * nz;
  const long long plane = (long long)nx * ny;
  const long long cell = z * plane + (long long)y * nx + x;
  const bool nr = x < nx && y < ny && near[x < nx && y < ny ? cell : 0] != 0;
  if (__any_sync(0xffffffffu, nr)) {
    const int xm = (x == 0) ? nx - 1 : x - 1, xp = (x + 1 >= nx) ? 0 : x + 1;
    const int ym = (y == 0) ? ny - 1 : y - 1, yp = (y + 1 >= ny) ? 0 : y + 1;
    const int zm = (z == 0) ? nz - 1 : z - 1, zp = (z + 1 >= nz) ? 0 : z + 1;
#pragma unroll
    for (int q = 1; q < Q; ++q) {
      const int cx = L::cx(q), cy = L::cy(q), cz = L::cz(q);
      const long long nb = (long long)(cz > 0 ? zp : (cz < 0 ? zm : z)) * plane +
                           (long long)(cy > 0 ? yp : (cy < 0 ? ym : y)) * nx + (cx > 0 ? xp : (cx < 0 ? xm : x));
      const bool link = nr && solid[nr ? nb : 0] != 0;
      double v = 0.0;
      if (link) {
        S s = f[(long long)q * n + cell] + f[(long long)L::opp(q) * n + nb];
        if (q_wall) {
          const float qw = q_wall[q_per_direction ? (long long)q * n + cell : cell];
          s = s * S(__fdiv_rn(1.0f, fmaxf(qw, 1e-6f)));
        }
        v = double(s);
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, link);
      if (ballot) {
        v = warp_sum(v);
        if ((threadIdx.x & 31) == 0) {
          atomicAdd(&acc[q], v);
          atomicAdd(&acc[Q + q], double(__popc(ballot)));
        }
      }
    }
  }
  __syncthreads();
  if (tid < 2 * Q && acc[tid] != 0.0) atomicAdd(&sums[tid], acc[tid]);
}

template <class L, typename S>
int launch_link_sums(const tlbm_desc* d, const void* f, const uint8_t* solid, const uint8_t* near,
                     const float* q_wall, int32_t q_per_direction, double* sums, cudaStream_t s) {
  dim3 grid, block;
  step_launch_shape(d->nx, d->ny, d->nz, grid, block);
  k_link_sums<L, S><<<grid, block, 0, s>>>(static_cast<const S*>(f), solid, near, q_wall, q_per_direction ? 1 : 0,
                                           d->nx, d->ny, d->nz, sums);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

}  // namespace
}  // namespace tlbm

using namespace tlbm;

extern "C" TLBM_API int tlbm_link_momentum_sums(const tlbm_desc* d, const void* f, const uint8_t* solid,
                                                const uint8_t* near, const float* q_wall,
                                                int32_t q_wall_per_direction, double* sums, void* stream) {
  if (!d || !f || !solid || !near || !sums) return TLBM_ERR_ARG;
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) return TLBM_ERR_SHAPE;
  if (d->nz > 65535 || (long long)d->nx * d->ny * d->nz > (1LL << 40)) return TLBM_ERR_SHAPE;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int q = d->lattice;
  if (q != TLBM_D2Q9 && q != TLBM_D3Q19 && q != TLBM_D3Q27) return TLBM_ERR_UNSUPPORTED;
  if (d->dtype != TLBM_F32 && d->dtype != TLBM_F64) return TLBM_ERR_DTYPE;
  if (cudaMemsetAsync(sums, 0, sizeof(double) * 2 * q, s) != cudaSuccess) return TLBM_ERR_LAUNCH;
#define TLBM_MEM(LAT)                                                                                             \
  return d->dtype == TLBM_F32                                                                                     \
             ? launch_link_sums<LAT, float>(d, f, solid, near, q_wall, q_wall_per_direction, sums, s)             \
             : launch_link_sums<LAT, double>(d, f, solid, near, q_wall, q_wall_per_direction, sums, s)
  if (q == TLBM_D2Q9) TLBM_MEM(D2Q9);
  if (q == TLBM_D3Q19) TLBM_MEM(D3Q19);
  TLBM_MEM(D3Q27);
#undef TLBM_MEM
}
