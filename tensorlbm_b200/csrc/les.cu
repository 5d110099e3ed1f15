// Learned LES closure: training-data kernels (filtered DNS moments, samples),
// the hand-written training step (forward + backward in fp32 on the CUDA
// cores, deterministic per-block gradient partials, Adam), weight packing for
// the tensor-core inference, and a stand-alone inference kernel.
#include <cuda_bf16.h>

#include "tlbm_collide.cuh"
#include "tlbm_mlp.cuh"

namespace tlbm {
namespace {

using mlp::H;
using mlp::NF;
using mlp::N_PARAMS;

// flat parameter offsets (the training vector)
constexpr int O_W1 = 0, O_B1 = O_W1 + H * NF, O_W2 = O_B1 + H, O_B2 = O_W2 + H * H, O_W3 = O_B2 + H,
              O_B3 = O_W3 + H * H, O_W4 = O_B3 + H, O_B4 = O_W4 + H;
static_assert(O_B4 + 1 == N_PARAMS, "parameter layout");

inline int launch_ok() { return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH; }

// ---------------------------------------------------------------------------
// filtered DNS moments: block means over factor^3 fine cells of
// rho, u, and u_i u_j (u the physical velocity m / rho (1 + A/2) of the
// exact-difference forcing)
// ---------------------------------------------------------------------------
__global__ void k_filter_moments(const float* __restrict__ f, int nx, int ny, int nz, int factor, float a_lin,
                                 float* __restrict__ out) {
  const int cx = nx / factor, cy = ny / factor, cz = nz / factor;
  const long long nc = (long long)cx * cy * cz;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int X = int(c % cx), Y = int((c / cx) % cy), Z = int(c / ((long long)cx * cy));
  const long long n = (long long)nx * ny * nz;
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double kf = 1.0 + 0.5 * double(a_lin);
  for (int dz = 0; dz < factor; ++dz)
    for (int dy = 0; dy < factor; ++dy)
      for (int dx = 0; dx < factor; ++dx) {
        const long long i = ((long long)(Z * factor + dz) * ny + (Y * factor + dy)) * nx + (X * factor + dx);
        double r = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
        for (int q = 0; q < D3Q19::Q; ++q) {
          const double v = f[(long long)q * n + i];
          r += v;
          mx += D3Q19::cx(q) * v;
          my += D3Q19::cy(q) * v;
          mz += D3Q19::cz(q) * v;
        }
        const double ux = mx / r * kf, uy = my / r * kf, uz = mz / r * kf;
        acc[0] += r;
        acc[1] += ux;
        acc[2] += uy;
        acc[3] += uz;
        acc[4] += ux * ux;
        acc[5] += uy * uy;
        acc[6] += uz * uz;
        acc[7] += ux * uy;
        acc[8] += ux * uz;
        acc[9] += uy * uz;
      }
  const double inv = 1.0 / double(factor * factor * factor);
#pragma unroll
  for (int k = 0; k < 10; ++k) out[(long long)k * nc + c] = float(acc[k] * inv);
}

// ---------------------------------------------------------------------------
// training samples of one filtered field (float64 arithmetic)
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long wrap_index(int x, int y, int z, int nx, int ny, int nz) {
  x = x < 0 ? x + nx : (x >= nx ? x - nx : x);
  y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
  z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
  return ((long long)z * ny + y) * nx + x;
}

__global__ void k_les_samples(const float* __restrict__ mom, int nx, int ny, int nz, double tau0, double c_s,
                              const float* __restrict__ nu_hat, float* __restrict__ x_out,
                              float* __restrict__ target, float* __restrict__ weight) {
  const long long n = (long long)nx * ny * nz;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = int(i % nx), y = int((i / nx) % ny), z = int(i / ((long long)nx * ny));
  auto u = [&](int comp, int xx, int yy, int zz) -> double {
    return mom[(long long)(1 + comp) * n + wrap_index(xx, yy, zz, nx, ny, nz)];
  };
  double g[3][3];  // g[i][j] = d_i u_j, periodic central differences
  for (int j = 0; j < 3; ++j) {
    g[0][j] = 0.5 * (u(j, x + 1, y, z) - u(j, x - 1, y, z));
    g[1][j] = 0.5 * (u(j, x, y + 1, z) - u(j, x, y - 1, z));
    g[2][j] = 0.5 * (u(j, x, y, z + 1) - u(j, x, y, z - 1));
  }
  const double s[6] = {g[0][0], g[1][1], g[2][2], 0.5 * (g[0][1] + g[1][0]), 0.5 * (g[0][2] + g[2][0]),
                       0.5 * (g[1][2] + g[2][1])};
  const double rho = mom[i];
  const double ux = mom[n + i], uy = mom[2 * n + i], uz = mom[3 * n + i];
  const double t[6] = {mom[4 * n + i] - ux * ux, mom[5 * n + i] - uy * uy, mom[6 * n + i] - uz * uz,
                       mom[7 * n + i] - ux * uy, mom[8 * n + i] - ux * uz, mom[9 * n + i] - uy * uz};
  const double ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  const double trt = (t[0] + t[1] + t[2]) / 3.0;
  const double tds = (t[0] - trt) * s[0] + (t[1] - trt) * s[1] + (t[2] - trt) * s[2] +
                     2.0 * (t[3] * s[3] + t[4] * s[4] + t[5] * s[5]);
  const double nu_star = -tds / (2.0 * ss + 1e-30);
  const double tau_eff = nu_hat ? tau0 + 3.0 * double(nu_hat[i]) : tau0 + 3.0 * c_s * c_s * sqrt(ss);
  const double k = -(2.0 / 3.0) * rho * tau_eff;
  double feat[NF];
  mlp::features<double>(k * s[0], k * s[1], k * s[2], k * s[3], k * s[4], k * s[5], rho, tau0, c_s, feat);
#pragma unroll
  for (int j = 0; j < NF; ++j) x_out[i * NF + j] = float(feat[j]);
  target[i] = float(nu_star);
  weight[i] = float(ss);
}

// ---------------------------------------------------------------------------
// training: forward + backward of a block of S samples, fp32
// ---------------------------------------------------------------------------
constexpr int S = 64;  // samples (threads) per block

__device__ __forceinline__ float sigm(float a) { return 1.0f / (1.0f + expf(-a)); }
__device__ __forceinline__ float silu_f(float a) { return a * sigm(a); }
__device__ __forceinline__ float dsilu_f(float a) {
  const float s = sigm(a);
  return s * (1.0f + a * (1.0f - s));
}
__device__ __forceinline__ float softplus_f(float y) { return fmaxf(y, 0.0f) + log1pf(expf(-fabsf(y))); }

struct TrainSmem {
  float w[N_PARAMS];
  float z[NF][S];
  float a1[H][S], a2[H][S], a3[H][S];
  float h1[H][S], h2[H][S];
  float g[H][S];
  float dy[S];
};

// One block = S samples idx[base .. base+S) of the (shuffled) index list.
// Writes the block's gradient of sum_s w_s (softplus(y_s) - t_s)^2 / batch and
// that loss to partial[block * (N_PARAMS + 1) ..].
__global__ void __launch_bounds__(S) k_mlp_grad(const float* __restrict__ theta, const float* __restrict__ mean,
                                                const float* __restrict__ istd, const float* __restrict__ x,
                                                const float* __restrict__ target, const float* __restrict__ weight,
                                                const long long* __restrict__ idx, long long count, float inv_batch,
                                                float* __restrict__ partial) {
  extern __shared__ __align__(16) uint8_t raw[];
  TrainSmem& sh = *reinterpret_cast<TrainSmem*>(raw);
  const int s = threadIdx.x;
  for (int p = s; p < N_PARAMS; p += S) sh.w[p] = theta[p];
  const long long gi = (long long)blockIdx.x * S + s;
  const bool live = gi < count;
  const long long row = live ? (idx ? idx[gi] : gi) : 0;
#pragma unroll
  for (int k = 0; k < NF; ++k) sh.z[k][s] = live ? (x[row * NF + k] - mean[k]) * istd[k] : 0.0f;
  __syncthreads();
  const float* W1 = sh.w + O_W1;
  const float* W2 = sh.w + O_W2;
  const float* W3 = sh.w + O_W3;
  // forward
  for (int j = 0; j < H; ++j) {
    float a = sh.w[O_B1 + j];
#pragma unroll
    for (int k = 0; k < NF; ++k) a = fmaf(W1[j * NF + k], sh.z[k][s], a);
    sh.a1[j][s] = a;
    sh.h1[j][s] = silu_f(a);
  }
  for (int j = 0; j < H; ++j) {
    float a = sh.w[O_B2 + j];
    for (int k = 0; k < H; ++k) a = fmaf(W2[j * H + k], sh.h1[k][s], a);
    sh.a2[j][s] = a;
    sh.h2[j][s] = silu_f(a);
  }
  float y = sh.w[O_B4];
  for (int j = 0; j < H; ++j) {
    float a = sh.w[O_B3 + j];
    for (int k = 0; k < H; ++k) a = fmaf(W3[j * H + k], sh.h2[k][s], a);
    sh.a3[j][s] = a;
    y = fmaf(sh.w[O_W4 + j], silu_f(a), y);
  }
  float loss = 0.0f, dy = 0.0f;
  if (live) {
    const float wgt = weight ? weight[row] : 1.0f;
    const float r = softplus_f(y) - target[row];
    loss = wgt * r * r * inv_batch;
    dy = 2.0f * wgt * r * inv_batch * sigm(y);
  }
  sh.dy[s] = dy;
  // G3[j][s] = dy w4[j] silu'(a3)
  for (int j = 0; j < H; ++j) sh.g[j][s] = dy * sh.w[O_W4 + j] * dsilu_f(sh.a3[j][s]);
  __syncthreads();
  float* out = partial + (long long)blockIdx.x * (N_PARAMS + 1);
  {
    // thread j: dw4[j], db3[j], dW3[j][:]
    const int j = s;
    float dw4 = 0.0f, db3 = 0.0f;
    for (int t = 0; t < S; ++t) {
      dw4 = fmaf(sh.dy[t], silu_f(sh.a3[j][t]), dw4);
      db3 += sh.g[j][t];
    }
    out[O_W4 + j] = dw4;
    out[O_B3 + j] = db3;
    for (int k = 0; k < H; ++k) {
      float acc = 0.0f;
      for (int t = 0; t < S; ++t) acc = fmaf(sh.g[j][t], sh.h2[k][t], acc);
      out[O_W3 + j * H + k] = acc;
    }
    if (j == 0) {
      float db4 = 0.0f;
      for (int t = 0; t < S; ++t) db4 += sh.dy[t];
      out[O_B4] = db4;
    }
  }
  // G2 = (W3^T G3) * silu'(a2), through registers
  {
    float g2[H];
    for (int k = 0; k < H; ++k) g2[k] = 0.0f;
    for (int j = 0; j < H; ++j) {
      const float gj = sh.g[j][s];
      for (int k = 0; k < H; ++k) g2[k] = fmaf(W3[j * H + k], gj, g2[k]);
    }
    __syncthreads();
    for (int k = 0; k < H; ++k) sh.g[k][s] = g2[k] * dsilu_f(sh.a2[k][s]);
  }
  __syncthreads();
  {
    const int j = s;
    float db2 = 0.0f;
    for (int t = 0; t < S; ++t) db2 += sh.g[j][t];
    out[O_B2 + j] = db2;
    for (int k = 0; k < H; ++k) {
      float acc = 0.0f;
      for (int t = 0; t < S; ++t) acc = fmaf(sh.g[j][t], sh.h1[k][t], acc);
      out[O_W2 + j * H + k] = acc;
    }
  }
  {
    float g1[H];
    for (int k = 0; k < H; ++k) g1[k] = 0.0f;
    for (int j = 0; j < H; ++j) {
      const float gj = sh.g[j][s];
      for (int k = 0; k < H; ++k) g1[k] = fmaf(W2[j * H + k], gj, g1[k]);
    }
    __syncthreads();
    for (int k = 0; k < H; ++k) sh.g[k][s] = g1[k] * dsilu_f(sh.a1[k][s]);
  }
  __syncthreads();
  {
    const int j = s;
    float db1 = 0.0f;
    for (int t = 0; t < S; ++t) db1 += sh.g[j][t];
    out[O_B1 + j] = db1;
    for (int k = 0; k < NF; ++k) {
      float acc = 0.0f;
      for (int t = 0; t < S; ++t) acc = fmaf(sh.g[j][t], sh.z[k][t], acc);
      out[O_W1 + j * NF + k] = acc;
    }
  }
  // block loss (fixed order over the block's samples)
  __syncthreads();
  sh.dy[s] = loss;
  __syncthreads();
  if (s == 0) {
    float l = 0.0f;
    for (int t = 0; t < S; ++t) l += sh.dy[t];
    out[N_PARAMS] = l;
  }
}

// sum the block partials in block order, then Adam (bias-corrected)
__global__ void k_mlp_adam(float* __restrict__ theta, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ partial, int nblocks, float lr, float b1, float b2, float eps,
                           float bc1, float bc2, float* __restrict__ grad_out, float* __restrict__ loss_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > N_PARAMS) return;
  float g = 0.0f;
  for (int b = 0; b < nblocks; ++b) g += partial[(long long)b * (N_PARAMS + 1) + p];
  if (p == N_PARAMS) {
    if (loss_out) *loss_out = g;
    return;
  }
  if (grad_out) grad_out[p] = g;
  if (lr == 0.0f) return;
  const float mm = b1 * m[p] + (1.0f - b1) * g;
  const float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  theta[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// fp32 forward of the training network (evaluation; same arithmetic as k_mlp_grad)
__global__ void __launch_bounds__(128) k_mlp_eval(const float* __restrict__ theta, const float* __restrict__ mean,
                                                  const float* __restrict__ istd, const float* __restrict__ x,
                                                  long long count, float* __restrict__ y_out) {
  __shared__ float w[N_PARAMS];
  for (int p = threadIdx.x; p < N_PARAMS; p += blockDim.x) w[p] = theta[p];
  __syncthreads();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float z[NF];
#pragma unroll
  for (int k = 0; k < NF; ++k) z[k] = (x[i * NF + k] - mean[k]) * istd[k];
  float h1[H], h2[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float a = w[O_B1 + j];
#pragma unroll
    for (int k = 0; k < NF; ++k) a = fmaf(w[O_W1 + j * NF + k], z[k], a);
    h1[j] = silu_f(a);
  }
#pragma unroll
  for (int j = 0; j < H; ++j) {
    float a = w[O_B2 + j];
#pragma unroll
    for (int k = 0; k < H; ++k) a = fmaf(w[O_W2 + j * H + k], h1[k], a);
    h2[j] = silu_f(a);
  }
  float y = w[O_B4];
#pragma unroll 4
  for (int j = 0; j < H; ++j) {
    float a = w[O_B3 + j];
#pragma unroll
    for (int k = 0; k < H; ++k) a = fmaf(w[O_W3 + j * H + k], h2[k], a);
    y = fmaf(w[O_W4 + j], silu_f(a), y);
  }
  y_out[i] = y;
}

// ---------------------------------------------------------------------------
// packing for the tensor-core inference
// ---------------------------------------------------------------------------
__global__ void k_mlp_pack(const float* __restrict__ theta, const float* __restrict__ mean,
                           const float* __restrict__ std, const float* __restrict__ lo, const float* __restrict__ hi,
                           float nu_scale, uint8_t* __restrict__ blob) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * H * H) {
    const int l = i / (H * H), n = (i / H) % H, k = i % H;
    float v;
    if (l == 0) v = k < NF ? theta[O_W1 + n * NF + k] : 0.0f;
    else v = theta[(l == 1 ? O_W2 : O_W3) + n * H + k];
    *reinterpret_cast<__nv_bfloat16*>(blob + mlp::OFF_W + l * mlp::W_TILE_BYTES + umma::sw128_offset(n, k)) =
        __float2bfloat16_rn(v);
  }
  if (i < H)  // output layer: row 0 of a 16-row tile (rows 1..15 stay zero)
    *reinterpret_cast<__nv_bfloat16*>(blob + mlp::OFF_W4 + umma::sw128_offset(0, i)) =
        __float2bfloat16_rn(theta[O_W4 + i]);
  if (i < mlp::P_COUNT) {
    float* p = reinterpret_cast<float*>(blob + mlp::OFF_P);
    float v = 0.0f;
    if (i < mlp::P_HB2) v = 0.5f * theta[O_B1 + i];  // hidden biases are stored halved
    else if (i < mlp::P_HB3) v = 0.5f * theta[O_B2 + i - mlp::P_HB2];
    else if (i < mlp::P_W4) v = 0.5f * theta[O_B3 + i - mlp::P_HB3];
    else if (i < mlp::P_B4) v = __bfloat162float(__float2bfloat16_rn(theta[O_W4 + i - mlp::P_W4]));
    else if (i == mlp::P_B4) v = theta[O_B4];
    else if (i == mlp::P_NUS) v = nu_scale;
    else if (i >= mlp::P_MEAN && i < mlp::P_ISTD) v = mean[i - mlp::P_MEAN];
    else if (i >= mlp::P_ISTD && i < mlp::P_LO) v = 1.0f / fmaxf(std[i - mlp::P_ISTD], 1e-6f);
    else if (i >= mlp::P_LO && i < mlp::P_HI) v = lo[i - mlp::P_LO];
    else if (i >= mlp::P_HI) v = hi[i - mlp::P_HI];
    p[i] = v;
  }
}

// stand-alone tensor-core inference: y for count raw feature rows
using InferCta = mlp::Cta<2>;

__global__ void __launch_bounds__(InferCta::THREADS)
    k_mlp_infer(const uint8_t* __restrict__ blob, const float* __restrict__ x, long long count,
                float* __restrict__ y_out, unsigned int* status) {
  extern __shared__ uint8_t raw[];
  mlp::Engine<2> e;
  e.setup(raw, blob);
  const float* p = e.params();
  const long long ntiles = (count + InferCta::THREADS - 1) / InferCta::THREADS;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const long long i = t * InferCta::THREADS + threadIdx.x;
    float z[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) z[k] = i < count ? (x[i * NF + k] - p[mlp::P_MEAN + k]) * p[mlp::P_ISTD + k] : 0.0f;
    bool ok = true;
    const float y = e.run(z, ok);
    if (i < count) y_out[i] = y;
    if (!ok) {  // uniform across the half
      if (e.lt == 0 && status) atomicOr(status, 4u);
      break;
    }
  }
  e.teardown();
}

int infer_grid(long long count, int& grid) {
  static int per_sm = -1, sms = 0;
  if (per_sm < 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TLBM_ERR_LAUNCH;
    if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, InferCta::SM_BYTES) !=
        cudaSuccess)
      return TLBM_ERR_LAUNCH;
    if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return TLBM_ERR_LAUNCH;
    per_sm = mlp::resident_ctas<2>(k_mlp_infer, sms);
  }
  if (per_sm < 1) return TLBM_ERR_UNSUPPORTED;
  const long long ntiles = (count + InferCta::THREADS - 1) / InferCta::THREADS;
  long long g = (long long)sms * per_sm;
  grid = int(g < ntiles ? g : ntiles);
  return TLBM_OK;
}

}  // namespace
}  // namespace tlbm

using namespace tlbm;

extern "C" {

TLBM_API int tlbm_les_filter_moments(const float* f, int32_t nx, int32_t ny, int32_t nz, int32_t factor,
                                     double a_lin, float* out, void* stream) {
  if (!f || !out) return TLBM_ERR_ARG;
  if (factor < 1 || nx < factor || ny < factor || nz < factor || nx % factor || ny % factor || nz % factor)
    return TLBM_ERR_SHAPE;
  const long long nc = (long long)(nx / factor) * (ny / factor) * (nz / factor);
  k_filter_moments<<<(unsigned)((nc + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      f, nx, ny, nz, factor, float(a_lin), out);
  return launch_ok();
}

TLBM_API int tlbm_les_samples(const float* moments, int32_t nx, int32_t ny, int32_t nz, double tau0, double c_s,
                              const float* nu_hat, float* features, float* target, float* weight, void* stream) {
  if (!moments || !features || !target || !weight) return TLBM_ERR_ARG;
  if (nx < 3 || ny < 3 || nz < 3) return TLBM_ERR_SHAPE;
  if (!(tau0 > 0.5)) return TLBM_ERR_ARG;
  const long long n = (long long)nx * ny * nz;
  k_les_samples<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      moments, nx, ny, nz, tau0, c_s, nu_hat, features, target, weight);
  return launch_ok();
}

TLBM_API int32_t tlbm_mlp_param_count(void) { return N_PARAMS; }
TLBM_API int32_t tlbm_mlp_blob_bytes(void) { return mlp::BLOB_BYTES; }
TLBM_API int64_t tlbm_mlp_grad_blocks(int64_t batch) { return (batch + S - 1) / S; }

TLBM_API int tlbm_mlp_grad(const float* theta, const float* mean, const float* istd, const float* x,
                           const float* target, const float* weight, const int64_t* idx, int64_t count,
                           float* partial, void* stream) {
  if (!theta || !mean || !istd || !x || !target || !partial) return TLBM_ERR_ARG;
  if (count < 1) return TLBM_ERR_SHAPE;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem)) !=
        cudaSuccess)
      return TLBM_ERR_LAUNCH;
    attr = true;
  }
  const long long blocks = (count + S - 1) / S;
  k_mlp_grad<<<(unsigned)blocks, S, sizeof(TrainSmem), static_cast<cudaStream_t>(stream)>>>(
      theta, mean, istd, x, target, weight, reinterpret_cast<const long long*>(idx), count, 1.0f / float(count),
      partial);
  return launch_ok();
}

TLBM_API int tlbm_mlp_adam(float* theta, float* m, float* v, const float* partial, int64_t nblocks, double lr,
                           double beta1, double beta2, double eps, int64_t step, float* grad_out, float* loss_out,
                           void* stream) {
  if (!theta || !m || !v || !partial) return TLBM_ERR_ARG;
  if (nblocks < 1 || step < 1) return TLBM_ERR_ARG;
  const float bc1 = float(1.0 - pow(beta1, double(step)));
  const float bc2 = float(1.0 - pow(beta2, double(step)));
  k_mlp_adam<<<(N_PARAMS + 1 + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      theta, m, v, partial, int(nblocks), float(lr), float(beta1), float(beta2), float(eps), bc1, bc2, grad_out,
      loss_out);
  return launch_ok();
}

TLBM_API int tlbm_mlp_eval(const float* theta, const float* mean, const float* istd, const float* x, int64_t count,
                           float* y, void* stream) {
  if (!theta || !mean || !istd || !x || !y) return TLBM_ERR_ARG;
  if (count < 1) return TLBM_OK;
  k_mlp_eval<<<(unsigned)((count + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(theta, mean, istd, x,
                                                                                             count, y);
  return launch_ok();
}

TLBM_API int tlbm_mlp_pack(const float* theta, const float* mean, const float* std, const float* lo, const float* hi,
                           double nu_scale, void* blob, void* stream) {
  if (!theta || !mean || !std || !lo || !hi || !blob) return TLBM_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(blob) % 16) return TLBM_ERR_ARG;
  if (cudaMemsetAsync(blob, 0, mlp::BLOB_BYTES, static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return TLBM_ERR_LAUNCH;
  k_mlp_pack<<<(3 * H * H + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      theta, mean, std, lo, hi, float(nu_scale), static_cast<uint8_t*>(blob));
  return launch_ok();
}

TLBM_API int tlbm_mlp_infer(const void* blob, const float* x, int64_t count, float* y, unsigned int* status,
                            void* stream) {
  if (!blob || !x || !y) return TLBM_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(blob) % 16) return TLBM_ERR_ARG;
  if (count < 1) return TLBM_OK;
  int grid = 0;
  int st = infer_grid(count, grid);
  if (st != TLBM_OK) return st;
  k_mlp_infer<<<grid, InferCta::THREADS, InferCta::SM_BYTES, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const uint8_t*>(blob), x, count, y, status);
  return launch_ok();
}

}  // extern "C"
