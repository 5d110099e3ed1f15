// Curved walls: Bouzidi (BFL) links of a sphere and the stand-alone link update.
//
// tlbm_sphere_links evaluates, per cell and direction, the test and the
// ray-sphere fraction of compute_q_sphere_common (bfl_common.py:384-477) in
// float64 with every operation rounded on its own (no contraction), in the
// order of the torch expressions, so the link mask and the float32 fractions
// are those of the reference bit for bit.  tlbm_bfl_bounce_back is
// bfl_bounce_back_common (bfl_common.py:106-190) on whole fields, with the
// force ledger of bouzidi_bounce_back_d3q19 (bfl_d3q19.py:339-377).
#include "tlbm_step.cuh"

namespace tlbm {
namespace {

__device__ __forceinline__ double sq(double v) { return __dmul_rn(v, v); }

// ((a - c)^2 summed over the three axes, left to right) for a point p + dc
__device__ __forceinline__ double dist2(double x, double y, double z, double dcx, double dcy, double dcz, double cx,
                                        double cy, double cz) {
  const double ex = __dsub_rn(__dadd_rn(x, dcx), cx), ey = __dsub_rn(__dadd_rn(y, dcy), cy),
               ez = __dsub_rn(__dadd_rn(z, dcz), cz);
  return __dadd_rn(__dadd_rn(sq(ex), sq(ey)), sq(ez));
}

template <class L>
__global__ void k_sphere_links(int nx, int ny, int nz, double cx, double cy, double cz, double radius,
                               uint8_t* __restrict__ mask, float* __restrict__ qf, uint8_t* __restrict__ solid) {
  const long long n = (long long)nx * ny * nz;
  const double r2 = sq(radius);
  for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < n;
       cell += (long long)gridDim.x * blockDim.x) {
    const int x = int(cell % nx), y = int((cell / nx) % ny), z = int(cell / ((long long)nx * ny));
    const double X = x, Y = y, Z = z;
    const double dx = __dsub_rn(X, cx), dy = __dsub_rn(Y, cy), dz = __dsub_rn(Z, cz);
    const bool fluid = __dadd_rn(__dadd_rn(sq(dx), sq(dy)), sq(dz)) > r2;
    if (solid) solid[cell] = fluid ? 0 : 1;
    mask[cell] = 0;
    qf[cell] = 0.5f;
#pragma unroll 1
    for (int d = 1; d < L::Q; ++d) {
      const double dcx = L::cx(d), dcy = L::cy(d), dcz = L::cz(d);
      const bool link = fluid && dist2(X, Y, Z, dcx, dcy, dcz, cx, cy, cz) <= r2;
      float q = 0.5f;
      if (link) {
        const double a = dcx * dcx + dcy * dcy + dcz * dcz;  // 1, 2 or 3, exact
        const double b = __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(dcx, dx), __dmul_rn(dcy, dy)),
                                                  __dmul_rn(dcz, dz)));
        const double c = __dsub_rn(__dadd_rn(__dadd_rn(sq(dx), sq(dy)), sq(dz)), r2);
        const double disc = __dsub_rn(sq(b), __dmul_rn(4.0 * a, c));
        const double root = __dsqrt_rn(disc >= 0.0 ? disc : 0.0);
        const double t1 = __ddiv_rn(__dsub_rn(-b, root), 2.0 * a);
        const double t2 = __ddiv_rn(__dadd_rn(-b, root), 2.0 * a);
        const bool v1 = (t1 > 1e-10) && (t1 <= 1.0 + 1e-10);
        const bool v2 = (t2 > 1e-10) && (t2 <= 1.0 + 1e-10);
        double fr = (v1 && v2) ? fmin(t1, t2) : (v1 ? t1 : (v2 ? t2 : 0.5));
        fr = fr < 1e-6 ? 1e-6 : (fr > 1.0 ? 1.0 : fr);
        q = __double2float_rn(fr);
      }
      mask[(long long)d * n + cell] = link ? 1 : 0;
      qf[(long long)d * n + cell] = q;
    }
  }
}

// One thread per cell: out[e] = value of link (x, opp e) where that link
// exists, f[e] elsewhere; the link's ledger term is warp-reduced into force.
template <class L, typename T>
__global__ void k_bfl_bounce_back(int nx, int ny, int nz, const T* __restrict__ f, const T* __restrict__ fp,
                                  const uint8_t* __restrict__ mask, const float* __restrict__ qf,
                                  T* __restrict__ out, double* force) {
  const long long n = (long long)nx * ny * nz;
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = cell < n;
  double mx = 0.0, my = 0.0, mz = 0.0;
  bool any = false;
  if (active) {
    const int x = int(cell % nx), y = int((cell / nx) % ny), z = int(cell / ((long long)nx * ny));
#pragma unroll 1
    for (int e = 0; e < L::Q; ++e) {
      const int dd = L::opp(e);
      T v = f[(long long)e * n + cell];
      if (mask[(long long)dd * n + cell]) {
        // P_d(x - c_d) with the periodic wrap of torch.roll
        const int ux = (x - L::cx(dd) + nx) % nx, uy = (y - L::cy(dd) + ny) % ny, uz = (z - L::cz(dd) + nz) % nz;
        const T pd = fp[(long long)dd * n + cell];
        const T up = fp[(long long)dd * n + ((long long)uz * ny + uy) * nx + ux];
        const T po = fp[(long long)e * n + cell];
        v = bfl_value(T(qf[(long long)dd * n + cell]), pd, up, po);
        const double s = double(xadd(pd, v));
        mx += L::cx(dd) * s;
        my += L::cy(dd) * s;
        mz += L::cz(dd) * s;
        any = true;
      }
      out[(long long)e * n + cell] = v;
    }
  }
  if (force) accumulate_force(force, __any_sync(0xffffffffu, any), mx, my, mz, 1.0);
}

int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return int(b < 148LL * 64 ? (b < 1 ? 1 : b) : 148LL * 64);
}

}  // namespace
}  // namespace tlbm

using namespace tlbm;

extern "C" {

TLBM_API int tlbm_sphere_links(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, double cx, double cy, double cz,
                               double radius, uint8_t* link_mask, float* q_field, uint8_t* solid, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1) return TLBM_ERR_SHAPE;
  if (!link_mask || !q_field || !(radius >= 0.0)) return TLBM_ERR_ARG;
  const long long n = (long long)nx * ny * nz;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (lattice == TLBM_D3Q19)
    k_sphere_links<D3Q19><<<blocks_for(n, 256), 256, 0, s>>>(nx, ny, nz, cx, cy, cz, radius, link_mask, q_field, solid);
  else if (lattice == TLBM_D3Q27)
    k_sphere_links<D3Q27><<<blocks_for(n, 256), 256, 0, s>>>(nx, ny, nz, cx, cy, cz, radius, link_mask, q_field, solid);
  else
    return TLBM_ERR_UNSUPPORTED;
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

TLBM_API int tlbm_bfl_bounce_back(const tlbm_desc* d, const void* f, const void* f_prev, const uint8_t* link_mask,
                                  const float* q_field, void* f_out, double* force, void* stream) {
  if (!d || !f || !f_prev || !link_mask || !q_field || !f_out) return TLBM_ERR_ARG;
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) return TLBM_ERR_SHAPE;
  if (f_out == f || f_out == f_prev) return TLBM_ERR_ALIAS;
  const long long n = (long long)d->nx * d->ny * d->nz;
  const int blocks = int((n + 255) / 256);
  if ((n + 255) / 256 > 0x7FFFFFFFLL) return TLBM_ERR_SHAPE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define TLBM_BFL(LAT, TY)                                                                                       \
  k_bfl_bounce_back<LAT, TY><<<blocks, 256, 0, s>>>(d->nx, d->ny, d->nz, static_cast<const TY*>(f),           \
                                                   static_cast<const TY*>(f_prev), link_mask, q_field,          \
                                                   static_cast<TY*>(f_out), force)
  if (d->lattice == TLBM_D3Q19 && d->dtype == TLBM_F32) TLBM_BFL(D3Q19, float);
  else if (d->lattice == TLBM_D3Q19 && d->dtype == TLBM_F64) TLBM_BFL(D3Q19, double);
  else if (d->lattice == TLBM_D3Q27 && d->dtype == TLBM_F32) TLBM_BFL(D3Q27, float);
  else if (d->lattice == TLBM_D3Q27 && d->dtype == TLBM_F64) TLBM_BFL(D3Q27, double);
  else return (d->lattice == TLBM_D3Q19 || d->lattice == TLBM_D3Q27) ? TLBM_ERR_DTYPE : TLBM_ERR_UNSUPPORTED;
#undef TLBM_BFL
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

}  // extern "C"
