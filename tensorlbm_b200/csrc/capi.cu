// extern "C" entry points (include/tlbm.h): argument checks, then dispatch to
// the typed kernels.  No entry point allocates or synchronises.
#include <atomic>
#include "ops.cuh"
#include "tlbm_aa.cuh"
#include "tlbm_dispatch.cuh"

using namespace tlbm;

namespace {

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline bool valid_lattice(int lattice) { return lattice == TLBM_D2Q9 || lattice == TLBM_D3Q19 || lattice == TLBM_D3Q27; }

// F32 / F64 only (the stand-alone operators mirror torch functions on float fields)
template <template <class, typename> class Fn, typename... A>
int by_lattice_real(int lattice, int dtype, A... a) {
  if (dtype != TLBM_F32 && dtype != TLBM_F64) return TLBM_ERR_DTYPE;
  const bool f64 = dtype == TLBM_F64;
  switch (lattice) {
    case TLBM_D2Q9: return f64 ? Fn<D2Q9, double>::run(a...) : Fn<D2Q9, float>::run(a...);
    case TLBM_D3Q19: return f64 ? Fn<D3Q19, double>::run(a...) : Fn<D3Q19, float>::run(a...);
    case TLBM_D3Q27: return f64 ? Fn<D3Q27, double>::run(a...) : Fn<D3Q27, float>::run(a...);
    default: return TLBM_ERR_UNSUPPORTED;
  }
}

template <class L, typename T> struct EqFn {
  static int run(long long n, const void* r, const void* a, const void* b, const void* c, void* o, cudaStream_t s) {
    return op_equilibrium<L, T>(n, r, a, b, c, o, s);
  }
};
template <class L, typename T> struct MacroFn {
  static int run(long long n, const void* f, void* r, void* a, void* b, void* c, cudaStream_t s) {
    return op_macroscopic<L, T>(n, f, r, a, b, c, s);
  }
};
template <class L, typename T> struct BbFn {
  static int run(long long n, const void* fi, const uint8_t* m, void* fo, cudaStream_t s) {
    return op_bounce_back<L, T>(n, fi, m, fo, s);
  }
};
template <class L, typename T> struct InletFn {
  static int run(int nx, int ny, int nz, void* f, double u, double uy, double uz, const void* px, const void* py,
                 cudaStream_t s) {
    return op_zou_he_inlet<L, T>(nx, ny, nz, f, u, uy, uz, px, py, s);
  }
};
template <class L, typename T> struct OutletFn {
  static int run(int nx, int ny, int nz, void* f, double rho, cudaStream_t s) {
    return op_zou_he_outlet<L, T>(nx, ny, nz, f, rho, s);
  }
};
template <class L, typename T> struct ForceFn {
  static int run(long long n, const void* f, const uint8_t* m, double* o, cudaStream_t s) {
    return op_obstacle_force<L, T>(n, f, m, o, s);
  }
};

bool shape_ok(int lattice, int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return false;
  if (lattice == TLBM_D2Q9 && nz != 1) return false;
  if (ny > 65535 || nz > 65535) return false;  // grid.y / grid.z limits of the step launch
  return true;
}

StepParams make_params(const tlbm_desc& d, const void* fin, void* fout, const uint8_t* flags, const float* tau_field,
                       double* force, unsigned int* status) {
  StepParams p;
  p.f_in = fin;
  p.f_out = fout;
  p.flags = flags;
  p.tau_field = tau_field;
  p.force = force;
  p.status = status;
  p.wall_velocity = d.wall_velocity;
  p.link_row = d.link_row;
  p.link_q = d.link_q;
  p.nx = d.nx;
  p.ny = d.ny;
  p.nz = d.nz;
  p.z0 = 0;
  p.z_count = d.nz;
  p.plane = (long long)d.nx * d.ny;
  p.n = p.plane * d.nz;
  p.bc = d.bc;
  p.tau = d.tau;
  p.inv_tau = 1.0 / d.tau;
  p.s_e = d.s_e;
  p.s_eps = d.s_eps;
  p.s_q = d.s_q;
  p.s_pi = d.s_pi;
  p.omega_b = d.omega_b;
  p.omega_odd = d.omega_odd;
  p.omega_even = d.omega_even;
  p.c_smag = d.c_smag;
  p.u_lid = d.u_lid;
  p.u_in[0] = d.u_in[0];
  p.u_in[1] = d.u_in[1];
  p.u_in[2] = d.u_in[2];
  p.rho_out = d.rho_out;
  return p;
}

int check_desc(const tlbm_desc* d) {
  if (!d) return TLBM_ERR_ARG;
  if (!valid_lattice(d->lattice)) return TLBM_ERR_UNSUPPORTED;
  if (!shape_ok(d->lattice, d->nx, d->ny, d->nz)) return TLBM_ERR_SHAPE;
  if (d->collision != TLBM_COLL_NONE && !(d->tau > 0.0)) return TLBM_ERR_ARG;
  if (d->collision == TLBM_COLL_TRT && !(d->tau > 0.5 && d->lambda_trt == d->lambda_trt)) return TLBM_ERR_ARG;
  if (d->collision == TLBM_COLL_CASCADED && !(d->tau > 0.5)) return TLBM_ERR_ARG;
  if ((d->bc & TLBM_BC_LID) && d->lattice == TLBM_D3Q27) return TLBM_ERR_UNSUPPORTED;
  if (d->bc & ~(uint32_t)(TLBM_BC_LID | TLBM_BC_ZH_INLET | TLBM_BC_ZH_OUTLET | TLBM_BC_FAR_FIELD | TLBM_BC_FAR_FIELD_Z))
    return TLBM_ERR_ARG;
  if (d->bc & (TLBM_BC_FAR_FIELD | TLBM_BC_FAR_FIELD_Z)) {
    // the far field owns the x planes; its z planes exist in 3-D only
    if (!(d->bc & TLBM_BC_FAR_FIELD) || (d->bc & (TLBM_BC_ZH_INLET | TLBM_BC_ZH_OUTLET)) || d->nx < 3 ||
        ((d->bc & TLBM_BC_FAR_FIELD_Z) && d->lattice == TLBM_D2Q9))
      return TLBM_ERR_ARG;
    for (int i = 0; i < 3; ++i)
      if (!(d->ff_inlet_du[i] == d->ff_inlet_du[i]) || !(d->u_in[i] == d->u_in[i])) return TLBM_ERR_ARG;
  }
  if (d->force_lin != 0.0) {
    if (!(d->force_lin == d->force_lin) || d->force_lin <= -1.0 || d->force_lin >= 1.0) return TLBM_ERR_ARG;
    if (d->collision != TLBM_COLL_BGK && d->collision != TLBM_COLL_MRT && d->collision != TLBM_COLL_SMAGORINSKY &&
        d->collision != TLBM_COLL_NONE)
      return TLBM_ERR_UNSUPPORTED;
  }
  return TLBM_OK;
}

int dispatch(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s) {
  switch (d.lattice) {
    case TLBM_D2Q9: return dispatch_step_d2q9(d, dtype_out, pull, p, s);
    case TLBM_D3Q19: return dispatch_step_d3q19(d, dtype_out, pull, p, s);
    case TLBM_D3Q27: return dispatch_step_d3q27(d, dtype_out, pull, p, s);
    default: return TLBM_ERR_UNSUPPORTED;
  }
}

int dispatch_aa_any(const tlbm_desc& d, int mode, const StepParams& p, cudaStream_t s) {
  switch (d.lattice) {
    case TLBM_D2Q9: return dispatch_aa_d2q9(mode, p, d, s);
    case TLBM_D3Q19: return dispatch_aa_d3q19(mode, p, d, s);
    case TLBM_D3Q27: return dispatch_aa_d3q27(mode, p, d, s);
    default: return TLBM_ERR_UNSUPPORTED;
  }
}

int check_aa(const tlbm_desc* d) {
  const int st = check_desc(d);
  if (st != TLBM_OK) return st;
  if (d->link_q || d->link_row || d->wall_velocity) return TLBM_ERR_UNSUPPORTED;
  // the far field's zero-gradient outlet reads the neighbour's post-stream
  // values, which the in-place AA steps do not keep
  if (d->bc & TLBM_BC_FAR_FIELD) return TLBM_ERR_UNSUPPORTED;
  if (d->dtype != TLBM_F32 && d->dtype != TLBM_F16_SHIFTED && d->dtype != TLBM_BF16_SHIFTED) return TLBM_ERR_DTYPE;
  return TLBM_OK;
}

}  // namespace

namespace tlbm {
namespace {
std::atomic<int> g_row_staging{0};
}
int row_staging_enabled() { return g_row_staging.load(std::memory_order_relaxed); }
int set_row_staging(bool enable) { return g_row_staging.exchange(enable ? 1 : 0); }
}  // namespace tlbm

extern "C" {

TLBM_API int tlbm_step(const tlbm_desc* d, const void* f_in, void* f_out, const uint8_t* flags,
                       const float* tau_field, double* force, unsigned int* status, void* stream) {
  int st = check_desc(d);
  if (st != TLBM_OK) return st;
  if (!f_in || !f_out) return TLBM_ERR_ARG;
  if (f_in == f_out) return TLBM_ERR_ALIAS;
  const StepParams p = make_params(*d, f_in, f_out, flags, tau_field, force, status);
  return dispatch(*d, d->dtype, true, p, as_stream(stream));
}

TLBM_API int tlbm_step_planes(const tlbm_desc* d, const void* f_in, void* f_out, const uint8_t* flags,
                              const float* tau_field, double* force, unsigned int* status, int32_t z_begin,
                              int32_t z_count, void* stream) {
  int st = check_desc(d);
  if (st != TLBM_OK) return st;
  if (!f_in || !f_out) return TLBM_ERR_ARG;
  if (f_in == f_out) return TLBM_ERR_ALIAS;
  if (z_begin < 0 || z_count < 1 || (long long)z_begin + z_count > d->nz) return TLBM_ERR_SHAPE;
  // z planes of a slab are not the domain's z faces
  if (d->bc & TLBM_BC_FAR_FIELD_Z) return TLBM_ERR_UNSUPPORTED;
  StepParams p = make_params(*d, f_in, f_out, flags, tau_field, force, status);
  p.z0 = z_begin;
  p.z_count = z_count;
  return dispatch(*d, d->dtype, true, p, as_stream(stream));
}

TLBM_API int tlbm_collide(const tlbm_desc* d, int32_t dtype_out, const void* f_in, void* f_out,
                          const uint8_t* flags, const float* tau_field, void* stream) {
  int st = check_desc(d);
  if (st != TLBM_OK) return st;
  if (!f_in || !f_out) return TLBM_ERR_ARG;
  if (f_in == f_out && dtype_out != d->dtype) return TLBM_ERR_ALIAS;
  tlbm_desc dd = *d;
  dd.bc = 0;
  const StepParams p = make_params(dd, f_in, f_out, flags, tau_field, nullptr, nullptr);
  return dispatch(dd, dtype_out, false, p, as_stream(stream));
}

TLBM_API int tlbm_stream(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, const void* f_in,
                         void* f_out, void* stream) {
  tlbm_desc d{};
  d.lattice = lattice;
  d.dtype = dtype;
  d.collision = TLBM_COLL_NONE;
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.tau = 1.0;
  return tlbm_step(&d, f_in, f_out, nullptr, nullptr, nullptr, nullptr, stream);
}

TLBM_API int tlbm_equilibrium(int32_t lattice, int32_t dtype, int64_t ncells, const void* rho, const void* ux,
                              const void* uy, const void* uz, void* f_out, void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!rho || !ux || !uy || !f_out || (lattice != TLBM_D2Q9 && !uz)) return TLBM_ERR_ARG;
  return by_lattice_real<EqFn>(lattice, dtype, (long long)ncells, rho, ux, uy, uz, f_out, as_stream(stream));
}

TLBM_API int tlbm_macroscopic(int32_t lattice, int32_t dtype, int64_t ncells, const void* f, void* rho, void* ux,
                              void* uy, void* uz, void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!f || !rho || !ux || !uy || (lattice != TLBM_D2Q9 && !uz)) return TLBM_ERR_ARG;
  return by_lattice_real<MacroFn>(lattice, dtype, (long long)ncells, f, rho, ux, uy, uz, as_stream(stream));
}

TLBM_API int tlbm_bounce_back(int32_t lattice, int32_t dtype, int64_t ncells, const void* f_in, const uint8_t* mask,
                              void* f_out, void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!f_in || !mask || !f_out) return TLBM_ERR_ARG;
  return by_lattice_real<BbFn>(lattice, dtype, (long long)ncells, f_in, mask, f_out, as_stream(stream));
}

TLBM_API int tlbm_moving_wall_bounce_back(int32_t lattice, int32_t dtype, int64_t ncells, const void* f_in,
                                          const uint8_t* mask, const void* wall_velocity, void* f_out,
                                          void* stream) {
  if (lattice != TLBM_D2Q9 && lattice != TLBM_D3Q19) return TLBM_ERR_UNSUPPORTED;
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!f_in || !mask || !wall_velocity || !f_out) return TLBM_ERR_ARG;
  if (dtype != TLBM_F32 && dtype != TLBM_F64) return TLBM_ERR_DTYPE;
  const bool f64 = dtype == TLBM_F64;
  cudaStream_t s = as_stream(stream);
  if (lattice == TLBM_D2Q9)
    return f64 ? op_moving_wall<D2Q9, double>(ncells, f_in, mask, wall_velocity, f_out, s)
               : op_moving_wall<D2Q9, float>(ncells, f_in, mask, wall_velocity, f_out, s);
  return f64 ? op_moving_wall<D3Q19, double>(ncells, f_in, mask, wall_velocity, f_out, s)
             : op_moving_wall<D3Q19, float>(ncells, f_in, mask, wall_velocity, f_out, s);
}

TLBM_API int tlbm_zou_he_inlet(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, void* f,
                               double u_in, double uy_in, double uz_in, const void* ux_profile,
                               const void* uy_profile, void* stream) {
  if (!valid_lattice(lattice)) return TLBM_ERR_UNSUPPORTED;
  if (!shape_ok(lattice, nx, ny, nz)) return TLBM_ERR_SHAPE;
  if (!f) return TLBM_ERR_ARG;
  if ((ux_profile || uy_profile) && lattice != TLBM_D2Q9) return TLBM_ERR_UNSUPPORTED;
  return by_lattice_real<InletFn>(lattice, dtype, (int)nx, (int)ny, (int)nz, f, u_in, uy_in, uz_in, ux_profile,
                                  uy_profile, as_stream(stream));
}

TLBM_API int tlbm_zou_he_outlet(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, void* f,
                                double rho_out, void* stream) {
  if (!valid_lattice(lattice)) return TLBM_ERR_UNSUPPORTED;
  if (!shape_ok(lattice, nx, ny, nz)) return TLBM_ERR_SHAPE;
  if (!f) return TLBM_ERR_ARG;
  return by_lattice_real<OutletFn>(lattice, dtype, (int)nx, (int)ny, (int)nz, f, rho_out, as_stream(stream));
}

TLBM_API int tlbm_moving_lid(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, void* f,
                             double u_lid, void* stream) {
  if (lattice != TLBM_D2Q9 && lattice != TLBM_D3Q19) return TLBM_ERR_UNSUPPORTED;
  if (!shape_ok(lattice, nx, ny, nz)) return TLBM_ERR_SHAPE;
  if (!f) return TLBM_ERR_ARG;
  if (dtype != TLBM_F32 && dtype != TLBM_F64) return TLBM_ERR_DTYPE;
  const bool f64 = dtype == TLBM_F64;
  cudaStream_t s = as_stream(stream);
  if (lattice == TLBM_D2Q9)
    return f64 ? op_moving_lid<D2Q9, double>(nx, ny, nz, f, u_lid, s) : op_moving_lid<D2Q9, float>(nx, ny, nz, f, u_lid, s);
  return f64 ? op_moving_lid<D3Q19, double>(nx, ny, nz, f, u_lid, s) : op_moving_lid<D3Q19, float>(nx, ny, nz, f, u_lid, s);
}

TLBM_API int tlbm_far_field(int32_t lattice, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, void* f,
                            double ux, double uy, double uz, int32_t z_faces, void* stream) {
  if (!valid_lattice(lattice)) return TLBM_ERR_UNSUPPORTED;
  if (!shape_ok(lattice, nx, ny, nz) || nx < 2) return TLBM_ERR_SHAPE;
  if (!f) return TLBM_ERR_ARG;
  if (dtype != TLBM_F32 && dtype != TLBM_F64) return TLBM_ERR_DTYPE;
  const bool f64 = dtype == TLBM_F64, zf = z_faces != 0 && lattice != TLBM_D2Q9;
  cudaStream_t s = as_stream(stream);
  switch (lattice) {
    case TLBM_D2Q9:
      return f64 ? op_far_field<D2Q9, double>(nx, ny, nz, f, ux, uy, uz, zf, s)
                 : op_far_field<D2Q9, float>(nx, ny, nz, f, ux, uy, uz, zf, s);
    case TLBM_D3Q19:
      return f64 ? op_far_field<D3Q19, double>(nx, ny, nz, f, ux, uy, uz, zf, s)
                 : op_far_field<D3Q19, float>(nx, ny, nz, f, ux, uy, uz, zf, s);
    default:
      return f64 ? op_far_field<D3Q27, double>(nx, ny, nz, f, ux, uy, uz, zf, s)
                 : op_far_field<D3Q27, float>(nx, ny, nz, f, ux, uy, uz, zf, s);
  }
}

TLBM_API int tlbm_obstacle_force(int32_t lattice, int32_t dtype, int64_t ncells, const void* f, const uint8_t* mask,
                                 double* out, void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!f || !mask || !out) return TLBM_ERR_ARG;
  return by_lattice_real<ForceFn>(lattice, dtype, (long long)ncells, f, mask, out, as_stream(stream));
}

TLBM_API int tlbm_correct_mass(int32_t dtype, int64_t count, const void* f_in, void* f_out, double target_mass,
                               double* scratch, void* stream) {
  if (count <= 0) return TLBM_ERR_SHAPE;
  if (!f_in || !f_out || !scratch) return TLBM_ERR_ARG;
  if (dtype == TLBM_F32) return op_correct_mass<float>(count, f_in, f_out, target_mass, scratch, as_stream(stream));
  if (dtype == TLBM_F64) return op_correct_mass<double>(count, f_in, f_out, target_mass, scratch, as_stream(stream));
  return TLBM_ERR_DTYPE;
}

TLBM_API int tlbm_moment_sums(int32_t lattice, int32_t dtype, int64_t ncells, const void* f, double* out,
                              void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!f || !out) return TLBM_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  const long long n = ncells;
#define TLBM_SUMS(L)                                                              \
  switch (dtype) {                                                                \
    case TLBM_F32: return op_moment_sums<L, float>(n, f, out, s);                 \
    case TLBM_F64: return op_moment_sums<L, double>(n, f, out, s);                \
    case TLBM_F16_SHIFTED: return op_moment_sums<L, __half>(n, f, out, s);        \
    case TLBM_BF16_SHIFTED: return op_moment_sums<L, __nv_bfloat16>(n, f, out, s); \
    default: return TLBM_ERR_DTYPE;                                               \
  }
  switch (lattice) {
    case TLBM_D2Q9: TLBM_SUMS(D2Q9)
    case TLBM_D3Q19: TLBM_SUMS(D3Q19)
    case TLBM_D3Q27: TLBM_SUMS(D3Q27)
    default: return TLBM_ERR_UNSUPPORTED;
  }
#undef TLBM_SUMS
}

TLBM_API int tlbm_sphere_mask(int32_t nx, int32_t ny, int32_t nz, double cx, double cy, double cz, double radius,
                              uint8_t* out, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return TLBM_ERR_SHAPE;
  if (!out) return TLBM_ERR_ARG;
  return op_sphere_mask(nx, ny, nz, cx, cy, cz, radius, out, as_stream(stream));
}

TLBM_API int tlbm_cylinder_mask(int32_t nx, int32_t ny, double cx, double cy, double radius, uint8_t* out,
                                void* stream) {
  if (nx <= 0 || ny <= 0) return TLBM_ERR_SHAPE;
  if (!out) return TLBM_ERR_ARG;
  return op_cylinder_mask(nx, ny, cx, cy, radius, out, as_stream(stream));
}

TLBM_API int tlbm_build_flags(int64_t ncells, const uint8_t* wall, const uint8_t* obstacle, uint32_t wall_flag,
                              uint8_t* flags, void* stream) {
  if (ncells <= 0) return TLBM_ERR_SHAPE;
  if (!flags) return TLBM_ERR_ARG;
  if (wall_flag != TLBM_FLAG_SOLID && wall_flag != TLBM_FLAG_HALFWAY) return TLBM_ERR_ARG;
  return op_build_flags(ncells, wall, obstacle, wall_flag, flags, as_stream(stream));
}

TLBM_API int tlbm_missing_mask(int32_t lattice, int32_t nx, int32_t ny, int32_t nz, const uint8_t* solid,
                               int32_t periodic_bits, uint8_t* missing, void* stream) {
  if (!valid_lattice(lattice)) return TLBM_ERR_UNSUPPORTED;
  if (nx <= 0 || ny <= 0 || nz <= 0 || (lattice == TLBM_D2Q9 && nz != 1)) return TLBM_ERR_SHAPE;
  if (!missing) return TLBM_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  switch (lattice) {
    case TLBM_D2Q9: return op_missing_mask<D2Q9>(nx, ny, nz, solid, periodic_bits, missing, s);
    case TLBM_D3Q19: return op_missing_mask<D3Q19>(nx, ny, nz, solid, periodic_bits, missing, s);
    default: return op_missing_mask<D3Q27>(nx, ny, nz, solid, periodic_bits, missing, s);
  }
}

TLBM_API int64_t tlbm_link_blocks(int64_t count) { return count <= 0 ? 0 : op_link_blocks(count); }

TLBM_API int tlbm_link_count(const uint8_t* mask, int64_t count, int64_t* block_counts, int64_t* count_out,
                             void* stream) {
  if (count < 0) return TLBM_ERR_SHAPE;
  if (!count_out || (count > 0 && (!mask || !block_counts))) return TLBM_ERR_ARG;
  return op_link_count(mask, count, (long long*)block_counts, (long long*)count_out, as_stream(stream));
}

TLBM_API int tlbm_link_list(const uint8_t* mask, int64_t count, const int64_t* block_counts, int64_t* out,
                            void* stream) {
  if (count < 0) return TLBM_ERR_SHAPE;
  if (count > 0 && (!mask || !block_counts || !out)) return TLBM_ERR_ARG;
  return op_link_list(mask, count, (const long long*)block_counts, (long long*)out, as_stream(stream));
}

TLBM_API const char* tlbm_status_string(int status) {
  switch (status) {
    case TLBM_OK: return "ok";
    case TLBM_ERR_SHAPE: return "invalid shape";
    case TLBM_ERR_DTYPE: return "unsupported dtype";
    case TLBM_ERR_ALIAS: return "input and output buffers alias";
    case TLBM_ERR_LAUNCH: return "CUDA launch failed";
    case TLBM_ERR_TIMEOUT: return "device wait timed out";
    case TLBM_ERR_NONFINITE: return "non-finite values";
    case TLBM_ERR_ARG: return "invalid argument";
    case TLBM_ERR_UNSUPPORTED: return "unsupported combination";
    case TLBM_ERR_TOO_LARGE: return "input exceeds the fixed static scratch of this allocation-free entry point";
    default: return "unknown status";
  }
}

TLBM_API int tlbm_abi_version(void) { return TLBM_ABI_VERSION; }

TLBM_API int tlbm_set_row_staging(int32_t enable) {
  return tlbm::set_row_staging(enable != 0);
}

TLBM_API int64_t tlbm_struct_size(int32_t which) {
  switch (which) {
    case 0: return (int64_t)sizeof(tlbm_desc);
    case 1: return (int64_t)sizeof(tlbm_batch_domain);
    case 2: return (int64_t)sizeof(tlbm_batch_desc);
    default: return -1;
  }
}

TLBM_API int tlbm_aa_load(const tlbm_desc* d, const void* f0, void* f, const uint8_t* flags, const float* tau_field,
                          void* stream) {
  const int st = check_aa(d);
  if (st != TLBM_OK) return st;
  if (!f0 || !f) return TLBM_ERR_ARG;
  if (f0 == f && d->dtype != TLBM_F32) return TLBM_ERR_ALIAS;
  tlbm_desc dd = *d;
  dd.bc = 0;
  const StepParams p = make_params(dd, f0, f, flags, tau_field, nullptr, nullptr);
  return dispatch_aa_any(dd, 2, p, as_stream(stream));
}

TLBM_API int tlbm_step_aa(const tlbm_desc* d, void* f, int32_t layout, const uint8_t* flags, const float* tau_field,
                          double* force, unsigned int* status, void* stream) {
  const int st = check_aa(d);
  if (st != TLBM_OK) return st;
  if (!f || layout < TLBM_AA_SWAPPED || layout > TLBM_AA_LOADED) return TLBM_ERR_ARG;
  const StepParams p = make_params(*d, f, f, flags, tau_field, force, status);
  const int mode = layout == TLBM_AA_SWAPPED ? 1 : (layout == TLBM_AA_NATURAL ? 0 : 5);
  return dispatch_aa_any(*d, mode, p, as_stream(stream));
}

TLBM_API int tlbm_aa_populations(const tlbm_desc* d, const void* f, int32_t layout, const uint8_t* flags,
                                 void* out, double* force, void* stream) {
  const int st = check_aa(d);
  if (st != TLBM_OK) return st;
  if (!f || !out || layout < TLBM_AA_SWAPPED || layout > TLBM_AA_LOADED) return TLBM_ERR_ARG;
  if (f == out) return TLBM_ERR_ALIAS;
  tlbm_desc dd = *d;
  dd.force_lin = 0.0;
  const StepParams p = make_params(dd, f, out, flags, nullptr, force, nullptr);
  const int mode = layout == TLBM_AA_SWAPPED ? 4 : (layout == TLBM_AA_NATURAL ? 3 : 6);
  return dispatch_aa_any(dd, mode, p, as_stream(stream));
}

}  // extern "C"
