/*
 * les_gpu.h -- C ABI of the B200 implementation of the paes-channelflow LES
 * per-timestep hot path (RK3 stage, x-y spectral derivatives, 3/2-dealiased
 * advection, SGS model, per-wavenumber tridiagonal pressure solve).
 *
 * The reference is a Fortran 90 program whose hot path is a set of
 * subroutines sharing module globals (modules.f90:1-61, compbuf.f90:1-32).
 * Each entry point below replaces one of those subroutines, keeps its
 * argument meaning, and works on a device-resident domain owned by an
 * opaque handle.  All functions return 0 on success or one of the LES_E*
 * codes; les_gpu_last_error() gives a readable message.  Signatures use
 * only plain C types so a Fortran bind(C) interface, ctypes, JNI or cgo can
 * bind them directly.
 *
 * Conventions
 *  - Layout: Fortran column-major (x fastest, then y, then z), levels
 *    iz = 1..nnz only (the halo levels of allocate.f90:14-36 are rebuilt on
 *    the device by les_gpu_lower / les_gpu_upper).
 *  - real_bytes selects 4 (shipped single-precision build) or 8
 *    (-fdefault-real-8 build) host arrays.
 *  - One CUDA stream per handle; calls are asynchronous except downloads,
 *    statistics and les_gpu_sync.  A handle is not re-entrant.
 */
#ifndef LES_GPU_H
#define LES_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (0 = success). */
#define LES_OK        0
#define LES_EINVAL    1  /* bad argument or configuration */
#define LES_ECUDA     2  /* CUDA runtime error */
#define LES_ENAN      3  /* NaN/Inf detected in the state */
#define LES_ETIMEOUT  4  /* bounded wait on the device expired */
#define LES_EUTAU     5  /* wall model blow-up guard: utau > 10 (lowerbc.f90:77-80) */
#define LES_ENOMEM    6  /* device allocation failed */
#define LES_ESTATE    7  /* entry points called out of order */
#define LES_ENOTBUILT 8  /* CUDA kernels unavailable (no device / not built) */

/* Sub-grid closure (parameters.f90:27-35 numbering for 3 and 4). */
#define LES_SGS_DEARDORFF 3  /* Moeng (1984) TKE model, imodel=3 */
#define LES_SGS_SMAG      4  /* Smagorinsky, imodel=4 */
#define LES_SGS_LEARNED   5  /* learned per-point closure with Deardorff fallback */

/* Precision forms. */
#define LES_PREC_FP64  8     /* plain FP64 drop-in */
#define LES_PREC_MIXED 4     /* FP32 transforms/advection/SGS, FP64 pressure and reductions */

/*
 * Run configuration: the namelist groups TIMING, GRIDSIZE and PARAMS of
 * les.F90:30-34 plus the hard-coded constants of les.F90:92-121 and
 * comp1.f90:152 made explicit.
 */
typedef struct les_config {
    int nnx, nny, nnz;      /* GRIDSIZE; nnx, nny even, of the form 2^a 3^b */
    int imodel;             /* LES_SGS_* */
    int isurface;           /* wall stress model 1..6 (lowerbc.f90:126-161) */
    int tke_production;     /* 0 = as shipped (no shear production), 1 = add xkk*shear */
    int precision;          /* LES_PREC_FP64 or LES_PREC_MIXED */
    int device;             /* CUDA device ordinal */
    double xl, yl, zl, z0;  /* PARAMS */
    double dt;              /* fixed time step (TIMING) */
    double cb, skc;         /* TIMING model constants (used only by derived c1..cnlin) */
    double nu;              /* molecular viscosity added to xkk (0 = reference physics) */
    double ugal, vgal;      /* Galilean shift of the wall model (0 in the reference) */
    double ufree;           /* sufsim floor on windm (uninitialised in the reference; 0) */
    double emin;            /* TKE floor, les.F90:102 (1e-6) */
    double forcing;         /* mean pressure gradient, comp1.f90:152 (0.016) */
} les_config;

typedef struct les_handle les_handle;

/* Fill *cfg with the reference defaults (default.f90, les.F90:92-121). */
void les_gpu_default_config(les_config* cfg);

/* Lifecycle: replaces setcombuf + allocate_arrays + initwave + fft_init
 * (les.F90:146-149, buffers.f90, allocate.f90:1-127, init.f90:4-44,
 * filter_fftw.f90:16-75). */
int  les_gpu_init(const les_config* cfg, les_handle** out);
/* Replaces fft_finalize + deallocate_arrays (les.F90:356-357). */
void les_gpu_finalize(les_handle* h);
const char* les_gpu_last_error(les_handle* h);

/* Host <-> device field transfer.  Upload replaces read_field + the deal()
 * of every level (read_write.f90:1-11, les.F90:185-190); the Nyquist modes of
 * u, v, w, e are removed on upload exactly as deal() does.  p is (nnx,nny,nnz).
 * Any pointer may be NULL to skip that field. */
int les_gpu_upload(les_handle* h, const void* u, const void* v, const void* w,
                   const void* e, const void* p, int real_bytes);
int les_gpu_download(les_handle* h, void* u, void* v, void* w, void* e, void* p,
                     int real_bytes);
/* Regridding (replaces the offline program redim.f90 plus the restart that
 * reads its output): dst's state (u, v, w, e, p) becomes src's state moved
 * onto dst's grid -- redim's linear z interpolation from src's levels
 * (interpol, redim.f90:202-269), spectral truncation / zero padding in x
 * and y (subroutine redim, redim.f90:277-318), e clamped to [1e-10, plane
 * maximum] (redim.f90:262-263), then the restart's deal of u, v, w, e
 * (les.F90:185-190) and w(nnz) = 0.  Both handles: same precision, device
 * and domain lengths (xl, yl, zl), else LES_EINVAL; any nnx, nny, nnz
 * each.  Synchronous; src is only read.  dst's tendencies are left as they
 * are (a restart starts a new RK3 step). */
int les_gpu_regrid(les_handle* dst, les_handle* src);
/* The tendencies ru, rv, rw, re (storage module, modules.f90:25-26). */
int les_gpu_upload_tendencies(les_handle* h, const void* ru, const void* rv,
                              const void* rw, const void* re, int real_bytes);
int les_gpu_download_tendencies(les_handle* h, void* ru, void* rv, void* rw,
                                void* re, int real_bytes);

/* Per-stage entry points, called in this order for istage = 1..3 exactly as
 * les.F90:254-285 calls the Fortran routines.
 *   les_gpu_lower   -> lower  (lowerbc.f90:1-20)
 *   les_gpu_upper   -> upper  (upperbc.f90:1-30)
 *   les_gpu_comp1   -> comp1  (comp1.f90:1-188) with derivs1/2, compadv1,
 *                      complen, compsgs1, compsgs3, sufsim, sufsim_upper,
 *                      expand/compress (filter_fftw.f90:254-308)
 *   les_gpu_comprhs -> comprhs (comprhs.f90:1-37)
 *   les_gpu_press   -> press   (press.F90:1-115) with tridv (tridv.f90)
 *   les_gpu_comp2   -> comp2   (comp2.f90:1-45)
 * dtab1 = dt*gama(istage), dtab2 = dt*zetas(istage), xkmax = dz*dz/dt/5
 * (les.F90:216, 255-257); mnout requests the stage-1 SGS means. */
int les_gpu_lower(les_handle* h);
int les_gpu_upper(les_handle* h);
int les_gpu_comp1(les_handle* h, int it, int mnout, int istage,
                  double dtab1, double dtab2, double xkmax);
int les_gpu_comprhs(les_handle* h, double dtabm);
int les_gpu_press(les_handle* h);
int les_gpu_comp2(les_handle* h, double dtab1);

/* One whole stage (lower, upper, comp1, comprhs, press, comp2) with the
 * fused kernels; identical results to the six calls above. */
int les_gpu_stage(les_handle* h, int it, int mnout, int istage,
                  double dtab1, double dtab2, double xkmax);
/* One RK3 step (three stages, les.F90:254-285) at time step dt, replayed
 * from a CUDA graph after the first call with the same (dt, mnout). */
int les_gpu_step(les_handle* h, int it, int mnout, double dt);

/* Statistics: compmn (compmn.F90:1-64) into meanbuf[19*nnz] (column-major
 * (19,nnz), rows in allocate.f90:89-111 order: englez, engsbz, divz, uxym,
 * vxym, wxym, uule, vvle, wwle, uwle, vwle, uvle, pple, uusb, vvsb, uvsb,
 * wwsb, uwsb, vwsb), all FP64.  scalars[5] = utau, utau_s, dudt, dvdt,
 * utau_lower (the values output_profiles prints, les.F90:389-407). */
int les_gpu_stats(les_handle* h, double* meanbuf, double* scalars);

/* 1D x-spectrum and ring-binned 2D spectrum of field `field` (0=u,1=v,2=w,
 * 3=e) at level iz (1-based): spectra (spectra2.f90:1-70).  Both outputs
 * have nnx/2+1 entries. */
int les_gpu_spectra(les_handle* h, int field, int iz, double* zspecx,
                    double* zspec2d);

/* Bounded wait for all queued work (LES_ETIMEOUT after timeout_s seconds);
 * also reads the device error word (NaN, utau guard). */
int les_gpu_sync(les_handle* h, double timeout_s);

/* Seeded synthetic initial condition built on the device: parabolic mean
 * u = 1.5*ub*(1-((z-h)/h)^2), i.i.d. uniform(-amp,amp)*utau perturbations of
 * u, v, w drawn from SplitMix64 streams seeded with seed+0,1,2 in
 * column-major order, e = e0, then deal() and one divergence projection
 * (comprhs + press + comp2 with dtab1 = 1).  Replaces initvel
 * (init.f90:50-114), whose same-seed-per-level recipe is not reproducible
 * across compilers. */
int les_gpu_make_ic(les_handle* h, unsigned long long seed, double ub,
                    double amp, double utau, double e0);

/* Advective CFL time step dt = cfl/max(ucfl,vcfl,wcfl,0.5/dz) of the current
 * state (les.F90:205-208). */
int les_gpu_cfl_dt(les_handle* h, double cfl, double* dt);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after the library's. */
void* les_gpu_stream(les_handle* h);

/* Number of kernels launched through this handle so far. */
long long les_gpu_kernel_launches(les_handle* h);

/* Tracing: run one stage (not graph-captured) with a CUDA event recorded
 * after every kernel on the handle's stream; ms[i] is the duration of the
 * i-th kernel and kernels[i] its host stub address (les_gpu_kernel_name
 * resolves it).  *nkernels receives the count; at most cap entries are
 * written.  Advances the state by one stage. */
int les_gpu_profile_stage(les_handle* h, int istage, double dt, double* ms,
                          const void** kernels, int cap, int* nkernels);

/* The device-side (mangled) name of the kernel whose host stub address is
 * `kernel` (as returned by les_gpu_profile_stage), NUL-terminated into
 * buf[cap]; kernels of internal linkage included.  LES_EINVAL for a NULL
 * argument or an address that is no kernel of this library. */
int les_gpu_kernel_name(const void* kernel, char* buf, int cap);

/* sizeof(les_config) as compiled into the library (binding sanity check). */
size_t les_gpu_config_size(void);

/* ---------------------------------------------------------------------
 * Operator-level entry points on caller-owned DEVICE buffers (FP64 or FP32
 * per real_bytes), enqueued on the caller's CUDA stream (NULL = legacy
 * default stream).  They expose the spectral core of filter_fftw.f90 and
 * tridv.f90 for unit testing and for callers that keep their own state.
 * Arrays are column-major (x fastest); `howmany` planes are processed.
 * --------------------------------------------------------------------- */

/* xderiv / yderiv (filter_fftw.f90:138-248): batched 1D spectral derivative
 * along x (y) with DC and Nyquist set to zero, planes of n1 x n2 with
 * domain lengths xl (yl). */
int les_op_xderiv(const void* ain, void* ax, int n1, int n2, int howmany,
                  double xl, int real_bytes, void* stream);
int les_op_yderiv(const void* ain, void* ay, int n1, int n2, int howmany,
                  double yl, int real_bytes, void* stream);
/* expand / compress / deal (filter_fftw.f90:254-329): 3/2 zero padding of
 * nx x ny planes onto (3nx/2) x (3ny/2) planes, truncation back, and
 * Nyquist removal. */
int les_op_expand(const void* xsmall, void* xlarge, int nx, int ny,
                  int howmany, int real_bytes, void* stream);
int les_op_compress(const void* xlarge, void* xsmall, int nx, int ny,
                    int howmany, int real_bytes, void* stream);
int les_op_deal(void* x, int nx, int ny, int howmany, int real_bytes,
                void* stream);
/* tridv (tridv.f90:1-55): bdar is (ny, n, 4) column-major holding the
 * sub-diagonal, diagonal, super-diagonal and right-hand side; the solution
 * overwrites bdar(:,:,4) and bdar(:,:,2) receives the inverted pivots, as
 * in the reference.  FP64 only (real_bytes = 8). */
int les_op_tridv(void* bdar, int ny, int n, int real_bytes, void* stream);

/* expand() without any device allocation.  It has no counterpart in the
 * reference.  Same arguments and results as les_op_expand, which allocates
 * its two scratch buffers per call; this variant keeps the scratch in a
 * static 16 MiB device array instead, for callers that must not allocate
 * device memory while they run (memory reserved up front by the host,
 * allocation-free regions, allocator policies that ban hidden allocations).
 * Limit: howmany*(nx/2)*(ny + 3*ny/2) complex values of scratch (16 bytes
 * each for real_bytes = 8, 8 for 4) must fit in 16 MiB, else LES_EINVAL.
 * Every device that loads the library keeps the array until exit; calls
 * share it, so calls that overlap on the GPU race; the first call on each
 * device does a one-time set-up and must come before any stream capture.
 * Under CUDA's lazy module loading (the default since CUDA 12.2) the array
 * is placed in device memory by that first call, not when the library is
 * loaded: a host that reserves all free device memory up front must make
 * its first call on each device before reserving, or run with
 * CUDA_MODULE_LOADING=EAGER. */
int les_op_expand_noalloc(const void* xsmall, void* xlarge, int nx, int ny,
                          int howmany, int real_bytes, void* stream);

/* Restart files (read_write.f90:16-40, les.F90:69-82 and 331-351): the
 * reference's Fortran unformatted sequential ".field" layout, each record
 * framed by its 4-byte length:
 *   time, nnx, nny, nnz, xl, yl, zl | dt, z0, utau |
 *   divgls, fcor, ugtop, ugbot, vgtop, vgbot | then per level iz = 1..nnz:
 *   u, v, w, e, p(1:nnx,1:nny) of level iz.
 * real_bytes: 4 for the shipped build, 8 for -fdefault-real-8 (integers are
 * 4 bytes in both).  Record 3 is not used by this path; it is written as
 * divgls = 0, fcor = 1e-4 (default.f90:23), ugtop = ugbot = 2 ugal and
 * vgtop = vgbot = 2 vgal, so that the post-processing programs' formula
 * ugal = (max(0, max(ugtop, ugbot)) + min(0, min(ugtop, ugbot))) / 2
 * (calc_pdf.f90:99-100) gives back the run's Galilean shift.
 *
 * les_gpu_write_field: downloads the state (synchronous on the device) and
 * writes the file; with async != 0 the file is written by a host thread and
 * the call returns once the data are on the host, so the handle can keep
 * stepping; les_gpu_field_wait joins that thread and returns its status (a
 * later write, read or finalize also waits for it).
 * les_gpu_read_field: reads a file of this handle's grid and uploads it
 * (upload semantics: deal, tendencies untouched); *time = its start time.
 * les_gpu_field_header: dims[3] and hdr[13] = time, xl, yl, zl, dt, z0,
 * utau, divgls, fcor, ugtop, ugbot, vgtop, vgbot without a handle. */
int les_gpu_write_field(les_handle* h, const char* path, double time, int real_bytes, int async);
int les_gpu_field_wait(les_handle* h);
int les_gpu_read_field(les_handle* h, const char* path, int real_bytes, double* time);
int les_gpu_field_header(const char* path, int real_bytes, int* dims, double* hdr);

/* Measurement helper with no counterpart in the reference: the device's
 * vector fused-multiply-add rate in flop/s for real_bytes = 4 (FP32) or 8
 * (FP64), timed by this library's own kernel (8 independent FMA chains per
 * thread, 16 CTAs of 256 threads per SM, CUDA events after a warm-up,
 * about 0.1 s).  It is the compute roof the FP32 / FP64 transform kernels
 * are read against.  Synchronous; allocates 8 bytes of device memory. */
int les_probe_fma_rate(int real_bytes, int device, double* flops_per_s);

/* Message of the last failed les_op_* call on this thread. */
const char* les_op_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* LES_GPU_H */
