/*
 * rtb.h -- C ABI of the B200 ray-tracing engine (librtb200.so).
 *
 * The library replaces the CUDA engine of amirych/rt behind the engine API of
 * common-lib/rt_engine_func.h:25-104.  Two families of entry points:
 *
 *  1. Drop-in calls (rtb_<reference name>): one per function of
 *     rt_engine_func.h, same arguments and semantics, host arrays in and out,
 *     synchronous.  rt_b200/shim/rt_engine_b200.cpp implements the reference's
 *     C++ prototypes on top of them, so Beam, Surface, TabulatedFunction,
 *     Scheme and ccd_frame link against this library unchanged.
 *  2. Device-resident calls (rtb_trace*, rtb_generate_beams, rtb_ccd_frame,
 *     rtb_adjoint_*): a whole scheme over many beams in one call, rays kept in
 *     HBM, asynchronous on a caller stream.
 *
 * Every function returns an int status: 0..4 equal RT_engine_error
 * (common-lib/rt_engine_errors.h:4-5); larger values name the exception the
 * reference would have thrown.  No function throws across the ABI.
 * Arrays are plain pointers; "host" arguments may be pageable or pinned
 * memory, "device" arguments must be device memory of the current device.
 */
#ifndef RTB_H
#define RTB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RTB_API __attribute__((visibility("default")))
#else
#define RTB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    RTB_OK = 0,               /* ENGINE_ERROR_OK */
    RTB_INIT_FAILED = 1,      /* ENGINE_ERROR_INIT_FAILED */
    RTB_BAD_ALLOC = 2,        /* ENGINE_ERROR_BAD_ALLOC */
    RTB_FAILED = 3,           /* ENGINE_ERROR_FAILED */
    RTB_BAD_VALUE = 4,        /* ENGINE_ERROR_BAD_VALUE */
    RTB_NO_INTERSECTIONS = 5, /* a stage lost every remaining ray (Surface::NoIntersections, surface.cpp:256,318) */
    RTB_NO_GOOD_RAYS = 6,     /* an action lost every remaining ray (Surface::NoGoodRays, surface.cpp:469,581) */
    RTB_OUT_OF_RANGE = 7      /* a wavelength outside a table (TabulatedFunction::OutOfRange, tabulated_function.cpp:179-181) */
};

/* ---- enumerations with the reference's numbering ------------------------ */
enum { RTB_PLANE = 0, RTB_CONIC = 1, RTB_TORIC = 2, RTB_AUX_CLASS = 3 };          /* surface.h:130 */
enum { RTB_MIRROR = 0, RTB_LENS = 1, RTB_GRATING = 2, RTB_STOP = 3,
       RTB_SHADE = 4, RTB_DETECTOR = 5, RTB_AUX_TYPE = 6 };                     /* surface.h:131 */
enum { RTB_CIRCLE = 0, RTB_RECTANGLE = 1 };                                    /* surface.h:132, beam.h:32 */
enum { RTB_REFLECTIVE = 0, RTB_TRANSPARENT = 1 };                              /* surface.h:241 */

/* ---- engine options ----------------------------------------------------- */
enum { RTB_ENGINE_PER_SURFACE = 0, RTB_ENGINE_FUSED = 1 };
/* RTB_FP64: the plain engine, IEEE FP64 (bit-exact with the reference's
 * arithmetic).  RTB_MIXED: FP64 ray state, FP32 surface normals, MUFU-seeded
 * divisions and square roots.  RTB_MIXED32: FP32 ray state and bulk
 * arithmetic (transforms, normals, reflection, refraction, renormalisation),
 * FP64 for the intersection roots, the grating equation and the detector
 * coordinate.  Both mixed engines are fused only; neither has a counterpart
 * in the reference, whose only scalar type is FP64 (num_defs.h:14). */
enum { RTB_FP64 = 0, RTB_MIXED = 1, RTB_MIXED32 = 2 };
/* Quirk fixes: 0 reproduces the reference; each bit selects the correct form. */
enum {
    RTB_FIX_TORIC_SIGN = 1,   /* iter_toric's 1+k1c^2Y^2 becomes 1-k1c^2Y^2 (cuda_engine/rt_cuda_engine_surface.cu:350) */
    RTB_FIX_TORIC_STEP = 2,   /* iter_toric's Steffensen step divides by Fzn-Fxn == 0 once converged and
                                 sends the ray to inf/NaN (surface.cu:390); the fix stops there instead */
    RTB_FIX_ASPHERE_ROOT = 4  /* iterative_conic/poly_intersection report the point before the last Newton
                                 update, up to 1e-7 mm short of the root (surface.cu:288-290); the fix reports
                                 the updated point */
};

#define RTB_MAX_POLY 10           /* MAX_POLY_COEFFS, surface.h:14 */
#define RTB_MAX_PARAMS 16         /* c, k, N, a1..a10, cR */
#define RTB_MAX_SURFACES 32
#define RTB_MAX_GRATINGS 8
#define RTB_MAX_KNOTS 1024
#define RTB_NOT_LOST 0xFF         /* lost_stage of a ray that reached the end */

/* A tabulated function (TabulatedFunction, tabulated_function.h:30-66):
 * n == 1 is a single value y[0] valid for any argument; n >= 4 knots x
 * strictly increasing with natural-spline second derivatives y2 (from
 * rtb_spline_init).  Pointers are host memory. */
typedef struct rtb_table {
    size_t n;
    const double* x;
    const double* y;
    const double* y2;
} rtb_table;

/* One surface, as Scheme::load_from_file builds it (common-lib/scheme.cpp:416-664). */
typedef struct rtb_surface {
    int32_t cls;                    /* RTB_PLANE .. RTB_AUX_CLASS */
    int32_t type;                   /* RTB_MIRROR .. RTB_AUX_TYPE */
    int32_t shape;                  /* RTB_CIRCLE / RTB_RECTANGLE */
    int32_t grating_type;           /* RTB_REFLECTIVE / RTB_TRANSPARENT */
    int64_t order;                  /* Grating::Order[0] (surface.h:277) */
    double gr_const;                /* grating constant, microns (surface.h:278) */
    double params[RTB_MAX_PARAMS];  /* Surface::Params: c, k, N, a1..aN [, cR] (surface.cpp:49-83) */
    double size[2];                 /* Surface::Size: radius, or width and height */
    double center[2];               /* Surface::Center */
    double distance[3];             /* Surface::Distance, mm */
    double angles_deg[3];           /* scheme angles, degrees, about y, x, z */
    rtb_table n1, n2;               /* refractive index before / after */
} rtb_surface;

/* One beam (one wavelength range of Scheme::run, scheme.cpp:966-1067): a
 * contiguous segment of the ray arrays plus what generates it. */
typedef struct rtb_beam {
    uint64_t first_ray;             /* index of the first ray in the ray arrays */
    uint64_t n_rays;
    int64_t orders[RTB_MAX_GRATINGS];  /* order of each grating in scheme order (range-file columns, scheme.cpp:1026-1032) */
    int32_t n_orders;               /* 0: every grating uses its own order */
    int32_t shape;                  /* RTB_CIRCLE (disk) */
    double disk[3];                 /* Beam::Params: rays per wavelength, R_in, R_out (beam.cpp:219-245) */
    double center[3];               /* Beam::Center */
    double range[2];                /* wavelength range, microns */
    uint64_t n_lambda;              /* composite beam: ray i takes lambda_(i mod n_lambda) (beam.cpp:470-484) */
    double field[2];                /* field angles, radians: direction (tan fx, tan fy, 1)/norm */
    uint64_t seed;                  /* Philox4x32-10 key of this beam's positions */
} rtb_beam;

/* Ray arrays (SoA, common-lib/beam.h:96-99).  Device memory for the
 * device-resident calls, host memory for rtb_trace_host. */
typedef struct rtb_rays {
    double *X, *Y, *Z, *cX, *cY, *cZ, *lambda;
    char* flag;                     /* 1 good, 0 lost */
    uint8_t* lost_stage;            /* 3*surface + {0 intersection, 1 aperture, 2 action}; RTB_NOT_LOST */
    size_t n;
} rtb_rays;

/* CCD geometry (ccd/ccd_frame.cpp:46-68): light-sensitive area in mm, pixel
 * counts, pixel size in mm. */
typedef struct rtb_ccd {
    double xsize, ysize;
    uint64_t xdim, ydim;
    double xpix, ypix;
} rtb_ccd;

/* The order in which a plan's fused kernel takes its rays (results do not
 * depend on it).  RTB_ORDER_COHERENT sorts the rays once, when the plan is
 * made, by beam, wavelength and Morton code of their entrance position, so
 * that a warp traces neighbouring rays of one wavelength, and keeps a copy of
 * the generated rays in that order, which the runs read (writes to the input
 * arrays rtb_plan_rays returns do not reach them; 62 bytes more per ray);
 * RTB_ORDER_INDEX takes the rays in index order from those arrays. */
enum { RTB_ORDER_COHERENT = 0, RTB_ORDER_INDEX = 1 };
/* Where a plan's fused kernel stores each ray's results: at the ray's index
 * (RTB_OUT_INDEX), or at its tracing slot (RTB_OUT_SLOT), so that the stores
 * of a warp are coalesced; rtb_plan_order gives the slot -> index map.  Frame
 * counts and statistics do not depend on it.  Traces other than plans store
 * at the index. */
enum { RTB_OUT_INDEX = 0, RTB_OUT_SLOT = 1 };

typedef struct rtb_trace_opts {
    int32_t engine;                 /* RTB_ENGINE_PER_SURFACE / RTB_ENGINE_FUSED */
    int32_t precision;              /* RTB_FP64 / RTB_MIXED / RTB_MIXED32 */
    uint32_t fixes;                 /* RTB_FIX_* bits */
    int32_t renormalize_lost;       /* apply the reference's trailing Normalize calls to lost rays (beam.cpp:527-571) */
    int32_t block_size;             /* 0: tuned default */
    int32_t rays_per_thread;        /* 0: tuned default */
    int32_t state_out;              /* fused: 1 writes X..cZ back, 0 writes only the CCD-plane X,Y */
    int32_t ray_order;              /* plans: RTB_ORDER_COHERENT (0) or RTB_ORDER_INDEX; other traces run in index order */
    const rtb_ccd* ccd;             /* optional: add good rays to frame counts (see rtb_ccd_frame) */
    uint32_t* counts;               /* device, ccd->xdim*ccd->ydim pixels; not cleared */
    uint64_t* n_outside;            /* device, may be NULL */
    int32_t out_order;              /* plans: RTB_OUT_INDEX (0) or RTB_OUT_SLOT */
    int32_t reserved;
} rtb_trace_opts;

/* Per-call statistics of a trace. */
typedef struct rtb_trace_stats {
    uint64_t ray_surfaces;          /* sum over rays of non-Aux surfaces reached (lost rays count their losing surface) */
    uint64_t n_good;                /* rays that reached the end */
    int32_t failed_beam;            /* first beam whose stage lost every remaining ray, -1 if none */
    int32_t failed_stage;           /* that stage, -1 if none */
} rtb_trace_stats;


/* =========================================================================
 * 1. Drop-in calls: rt_engine_func.h, host arrays, synchronous.
 * ========================================================================= */

/* rt_engine_init (rt_engine_func.h:25): selects device 0, creates the stream
 * and the device arena.  Idempotent. */
RTB_API int rtb_init(void);

/* rt_engine_info (rt_engine_func.h:26): newline-separated info lines into buf. */
RTB_API int rtb_info(char* buf, size_t buflen);

/* beam_random (rt_engine_func.h:30-31): uniform disk, params = [N, R_in, R_out],
 * center = [x, y, z].  Positions come from Philox4x32-10 keyed by `seed`, ray
 * `first_ray + i`, in place of the reference's clock-seeded cuRAND. */
RTB_API int rtb_beam_random(int shape, const double* params, const double* center, size_t n,
                    double* X, double* Y, double* Z, uint64_t seed, uint64_t first_ray);

/* beam_conic_cosins (rt_engine_func.h:33); conic_angle in radians. */
RTB_API int rtb_beam_conic_cosins(size_t n, double conic_angle, const double* X, const double* Y,
                          double* cX, double* cY, double* cZ);

/* beam_gauss_cosins (rt_engine_func.h:35); fwhm in arcsec. */
RTB_API int rtb_beam_gauss_cosins(size_t n, double fwhm, double* cX, double* cY, double* cZ, uint64_t seed);

/* uniform_range_beam (rt_engine_func.h:37). */
RTB_API int rtb_uniform_range_beam(size_t n, const double* range, double* lambda);

/* random_range_beam (rt_engine_func.h:39). */
RTB_API int rtb_random_range_beam(size_t n, const double* range, double* lambda, uint64_t seed);

/* beam_transform (rt_engine_func.h:41-42); angles in radians. */
RTB_API int rtb_beam_transform(size_t n, const double* angles, const double* dist,
                       double* X, double* Y, double* Z, double* cX, double* cY, double* cZ);

/* surface_intersection (rt_engine_func.h:46-49).  *n_bad is incremented. */
RTB_API int rtb_surface_intersection(int cls, const double* params, size_t n,
                             double* X, double* Y, double* Z, double* cX, double* cY, double* cZ,
                             size_t* n_bad, char* flag);
/* surface_intersection with quirk fixes (RTB_FIX_* bits); no reference counterpart. */
RTB_API int rtb_surface_intersection_fix(int cls, const double* params, size_t n, double* X, double* Y, double* Z,
                                         double* cX, double* cY, double* cZ, size_t* n_bad, char* flag,
                                         uint32_t fixes);

/* surface_reflection (rt_engine_func.h:52-54). */
RTB_API int rtb_surface_reflection(int cls, const double* params, size_t n,
                           double* X, double* Y, double* Z, double* cX, double* cY, double* cZ);

/* surface_refraction (rt_engine_func.h:57-61). */
RTB_API int rtb_surface_refraction(int cls, const double* params, size_t n,
                           double* X, double* Y, double* Z, double* cX, double* cY, double* cZ,
                           const double* lambda, const rtb_table* n1, const rtb_table* n2,
                           size_t* n_bad, char* flag);

/* surface_diffration (rt_engine_func.h:64-70). */
RTB_API int rtb_surface_diffration(int cls, int gr_type, const double* params, long diff_order,
                           double gr_constant, size_t n,
                           double* X, double* Y, double* Z, double* cX, double* cY, double* cZ,
                           const double* lambda, const rtb_table* n1, const rtb_table* n2,
                           size_t* n_bad, char* flag);

/* surface_QE (rt_engine_func.h:73): spec[i] *= QE(lambda[i]). */
RTB_API int rtb_surface_QE(size_t n, const double* lambda, double* spec, const rtb_table* qe);

/* grating_energy_distr (rt_engine_func.h:75-78); angles in radians. */
RTB_API int rtb_grating_energy_distr(size_t n, const double* lambda, long order, double blaze_angle,
                             double alpha, double gamma, double gr_const, double rule_start,
                             double rule_stop, double* energy_distr);

/* rt_engine_free_vector / rt_engine_alocate_vector (rt_engine_func.h:84-86):
 * page-locked host vectors, so the drop-in copies run at full PCIe rate. */
RTB_API void rtb_free_vector(double* data);
RTB_API double* rtb_alocate_vector(size_t n_elem);

/* spline_init (rt_engine_func.h:91): natural cubic spline second derivatives. */
RTB_API int rtb_spline_init(size_t n, const double* x, const double* y, double* y2);

/* ccd_coordinates (rt_engine_func.h:96-99). */
RTB_API int rtb_ccd_coordinates(size_t n, const double* X, const double* Y, double ccd_xsize,
                        double ccd_ysize, double ccd_xpix, double ccd_ypix,
                        unsigned int* ccd_X, unsigned int* ccd_Y);

/* compute_ccd_image (rt_engine_func.h:101-104): image += spec(l)*l/hc*QE(l)*pix_area
 * per ray; rays whose pixel lies outside xdim x ydim are skipped and counted
 * in *n_outside (may be NULL). */
RTB_API int rtb_compute_ccd_image(size_t n, const unsigned int* ccd_X, const unsigned int* ccd_Y,
                          const double* lambda, const rtb_table* qe, const rtb_table* spec,
                          size_t xdim, size_t ydim, double xpix, double ypix, double* image,
                          uint64_t* n_outside);

/* Host loops of Beam and Surface run on the device.
 * Beam::Normalize (beam.cpp:527-571). */
RTB_API int rtb_normalize(size_t n, double* cX, double* cY, double* cZ);
/* Surface::ApplyConstrains / Shade::ApplyConstrains (surface.cpp:264-321,652-699);
 * shade != 0 selects the inverted test.  *n_bad is incremented. */
RTB_API int rtb_apply_constrains(int shade, int shape, const double* size, const double* center, size_t n,
                         const double* X, const double* Y, char* flag, size_t* n_bad);
/* Beam::Rearrange (beam.cpp:574-598) over the good prefix [0, *n_good) of the
 * seven arrays; *n_good is updated. */
RTB_API int rtb_rearrange(size_t* n_good, double* X, double* Y, double* Z, double* cX, double* cY,
                  double* cZ, double* lambda, char* flag);

/* =========================================================================
 * 2. Device-resident calls.  `stream` is a cudaStream_t (NULL: the library's
 *    own stream).  Each call is ordered on that stream.
 * ========================================================================= */

/* Fill rays[first_ray, first_ray+n_rays) of every beam: uniform disk positions
 * (Philox4x32-10), parallel cosines turned by the field angles, composite
 * uniform wavelengths, flag 1, lost_stage RTB_NOT_LOST. */
RTB_API int rtb_generate_beams(const rtb_beam* beams, size_t n_beams, const rtb_rays* rays, void* stream);

/* Trace every beam through the scheme, in place (Scheme::run's per-surface
 * loop, scheme.cpp:983-1055).  Rays keep their index; lost rays carry
 * flag 0 and lost_stage.  stats may be NULL. */
RTB_API int rtb_trace(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
              const rtb_trace_opts* opts, const rtb_rays* rays, rtb_trace_stats* stats, void* stream);

/* rtb_trace reading `in` and writing `out` (in may equal out).  `in` keeps
 * its contents; out->lambda is not written.  With opts->state_out == 0 only
 * X, Y, flag and lost_stage of `out` are written. */
RTB_API int rtb_trace_out(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                          const rtb_trace_opts* opts, const rtb_rays* in, const rtb_rays* out,
                          rtb_trace_stats* stats, void* stream);

/* rtb_trace_out for callers that cannot allocate memory (no counterpart in
 * the reference).  Runs the fused kernel (opts->engine must be
 * RTB_ENGINE_FUSED; block_size and rays_per_thread as rtb_trace_out takes
 * them) with its scratch -- prepared scheme, tables, beam table, loss
 * counters -- in a file-scope device array of RTB_NOALLOC_SCRATCH_BYTES per
 * device and host-side staging in file-scope host arrays: no cudaMalloc,
 * cudaFree, pool or heap allocation.  Requests that do not fit (more than
 * RTB_NOALLOC_MAX_KNOTS table values, too many beams x stages for the
 * counters, or more shared memory than a block may have) return
 * RTB_BAD_VALUE before any work is queued; with the largest tables the array
 * holds the counters of 1,100 beams of a 32-surface scheme.  The first call
 * on a device looks up the array's address with that device current.  A NULL
 * stream (the library's own) is valid only
 * on the device the library was first used on.  Calls run one at a time and
 * each returns with `stream` synchronised; all calls share the array, so
 * other GPU work that wrote it during a call would race with that call. */
#define RTB_NOALLOC_SCRATCH_BYTES 1048576
#define RTB_NOALLOC_MAX_KNOTS 8192
RTB_API int rtb_trace_out_noalloc(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams,
                                  size_t n_beams, const rtb_trace_opts* opts, const rtb_rays* in,
                                  const rtb_rays* out, rtb_trace_stats* stats, void* stream);

/* rtb_trace on host arrays: copies in, traces and copies out, overlapping the
 * copies of one chunk with the trace of another.  Synchronous. */
RTB_API int rtb_trace_host(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams,
                   size_t n_beams, const rtb_trace_opts* opts, const rtb_rays* host_rays,
                   rtb_trace_stats* stats);

/* Fault hook for tests (no reference counterpart): after the library's next
 * `after` device allocations, the `count` following ones fail as if the
 * device were out of memory, so that the calls making them return
 * RTB_BAD_ALLOC (the reference's ENGINE_ERROR_BAD_ALLOC,
 * rt_engine_errors.h:4) and release what they had allocated.  count 0
 * clears it. */
RTB_API int rtb_fail_allocations(uint32_t after, uint32_t count);

/* Frame counts: counts[iy*xdim + ix] += 1 for every good ray whose pixel
 * (ccd_coordinates, ccd.cu:30-45) lies on the CCD; *n_outside (device, may be
 * NULL) counts the good rays that do not.  counts is not cleared. */
RTB_API int rtb_ccd_frame(const rtb_rays* rays, const rtb_ccd* ccd, uint32_t* counts, uint64_t* n_outside,
                  void* stream);

/* Order of the rays as the reference's Rearrange calls leave them
 * (beam.cpp:574-598), from lost_stage: order[k] is the index of the ray at
 * position k of the reference's arrays for beam b; positions [0, n_good) are
 * the good rays.  order is device memory of rays->n entries. */
RTB_API int rtb_reference_order(const rtb_beam* beams, size_t n_beams, size_t n_stages, const rtb_rays* rays,
                        uint32_t* order, void* stream);

/* =========================================================================
 * 3. Plans: many beams of uneven size, wavelength, field angle and order
 *    traced by one graph launch, with a launch-configuration autotuner.  No
 *    counterpart in the reference; Scheme::run's loop over ranges
 *    (scheme.cpp:983-1055) maps to one plan whose beams are the ranges.
 *    A plan is used by one host thread at a time.
 * ========================================================================= */
typedef struct rtb_plan rtb_plan;

/* One measured launch configuration (rtb_plan_autotune). */
typedef struct {
    int32_t block_size;      /* threads per block */
    int32_t rays_per_thread; /* a warp takes tiles of 32 x rays_per_thread rays */
    double ms;               /* mean device time of one run */
} rtb_tune_entry;

/* Prepare a plan on the current device: the scheme and the beam table in
 * device memory, the rays of all beams generated once (as
 * rtb_generate_beams), output arrays, the loss counters and page-locked host
 * copies of them.  opts is copied; opts->engine must be RTB_ENGINE_FUSED.
 * When opts->ccd and opts->counts are set, every run adds its good rays to
 * that frame (the plan never clears it).  block_size / rays_per_thread 0
 * take the configuration an earlier rtb_plan_autotune chose for the same
 * scheme, precision, frame use and ray count in this process, else the
 * defaults (256 x 2).  A plan launches a copy of the fused kernel of its
 * precision compiled for its scheme's structure with NVRTC when the plan is
 * made (the same arithmetic -- for RTB_FP64 the same IEEE operations, bit
 * for bit -- without the per-surface branching on surface kind, type and
 * shape; cached per structure for the process), unless RTB_SPECIALIZE=0 is
 * set in the environment or NVRTC is unavailable; see rtb_plan_specialized.
 * No counterpart in the reference, which has no fused kernel. */
RTB_API int rtb_plan_create(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                            const rtb_trace_opts* opts, rtb_plan** plan);
/* One trace of the plan's rays as a CUDA graph launched on `stream` (NULL:
 * the plan's own stream): clear the counters, run the fused kernel, copy the
 * counters to the host.  The graph is captured on the first run and again
 * after the launch configuration changes.  Asynchronous.  The generated rays
 * are read, not modified; results go to the plan's output arrays. */
RTB_API int rtb_plan_run(rtb_plan* plan, void* stream);
/* Waits for the last run; its status and statistics as rtb_trace returns them
 * (RTB_NO_INTERSECTIONS / RTB_NO_GOOD_RAYS name the first beam that lost
 * every ray; the other beams are traced all the same). */
RTB_API int rtb_plan_result(rtb_plan* plan, rtb_trace_stats* stats);
/* Per-(beam, stage) counters of the last run, as rtb_trace_opts.counts
 * describes them: counts[b * (3 * n_surfaces + 1) + s] rays of beam b lost at
 * stage s (3 per surface: intersection, aperture, action), then the rays of
 * beam b that reached the end.  Waits for the last run.  capacity is in
 * entries; *n_entries (may be NULL) receives the number available. */
RTB_API int rtb_plan_counts(rtb_plan* plan, uint64_t* counts, size_t capacity, size_t* n_entries);
/* Device arrays of the plan: `in` the generated rays, `out` the output of the
 * last run (X, Y, flag, lost_stage; every state array with opts->state_out;
 * out->lambda is in->lambda).  Either may be NULL. */
RTB_API int rtb_plan_rays(const rtb_plan* plan, rtb_rays* in, rtb_rays* out);
/* The plan's tracing order (device, n_rays entries: slot -> ray index), or
 * NULL for a plan in index order (slot == index).  With RTB_OUT_SLOT, output
 * slot s holds the results of ray order[s].  No reference counterpart. */
RTB_API int rtb_plan_order(const rtb_plan* plan, const uint32_t** order);
/* Time block_size {128, 256, 512 (RTB_MIXED only)} x rays_per_thread
 * {1, 2, 4, 8}: one untimed run, then `reps` runs, each configuration into a
 * private frame so the plan's frame is untouched.  The fastest becomes the
 * plan's configuration and the one later plans of the same key start with.
 * table (capacity entries, may be NULL) receives the measurements,
 * *n_entries (may be NULL) their number.  Synchronous. */
RTB_API int rtb_plan_autotune(rtb_plan* plan, int reps, rtb_tune_entry* table, size_t capacity, size_t* n_entries);
/* Set the launch configuration explicitly (RTB_BAD_VALUE if unsupported). */
RTB_API int rtb_plan_set_config(rtb_plan* plan, int32_t block_size, int32_t rays_per_thread);
/* The plan's launch configuration and ray count. */
RTB_API int rtb_plan_config(const rtb_plan* plan, int32_t* block_size, int32_t* rays_per_thread, uint64_t* n_rays);
/* *specialized = 1 when the plan launches a kernel compiled for its scheme,
 * else 0; note (may be NULL, note_len bytes) receives why not ("" when
 * specialised). */
RTB_API int rtb_plan_specialized(const rtb_plan* plan, int32_t* specialized, char* note, size_t note_len);
/* Compile the fused kernel of `precision` (RTB_FP64 / RTB_MIXED) specialised
 * to this scheme's structure ahead of rtb_plan_create (which compiles it
 * otherwise, once per structure and process); needs no device.  Once
 * compiled, one-shot fused traces of that precision and a scheme of that
 * structure (rtb_trace, rtb_trace_out, rtb_trace_host) launch it too; they
 * never compile it themselves.  RTB_OK when compiled; RTB_FAILED with the
 * reason in note (may be NULL) when NVRTC is unavailable or fails.  With
 * RTB_JIT_CACHE=<directory> in the environment, compiled kernels are also
 * kept in files there and later processes load them instead of compiling.
 * No counterpart in the reference. */
RTB_API int rtb_specialize(const rtb_surface* surfaces, size_t n_surfaces, uint32_t fixes, int32_t precision,
                           char* note, size_t note_len);
/* Release everything the plan holds, after its work has finished. */
RTB_API int rtb_plan_destroy(rtb_plan* plan);

/* =========================================================================
 * 5. Scheme files: the reference's scheme XML (Scheme::load_from_file,
 *    common-lib/scheme.cpp:272-857) read without Mini-XML.  Values are element
 *    texts; n1/n2 and the beam range may name files (two-column tables of at
 *    least 4 rows; range rows "w1 w2 order_1 .. order_G"), looked up relative
 *    to the working directory as the reference does, then to the scheme
 *    file's directory.  Surfaces are taken in document order.
 * ========================================================================= */
enum { RTB_BEAM_PARALLEL = 0, RTB_BEAM_CONIC = 1, RTB_BEAM_GAUSS = 2 };          /* beam.h:31 */
enum { RTB_PROFILE_RANDOM = 0, RTB_PROFILE_CONCENTRIC = 1 };                      /* beam.h:33 */
enum { RTB_RANGE_RANDOM = 0, RTB_RANGE_UNIFORM = 1, RTB_RANGE_MONOCHROMATIC = 2 }; /* beam.h:34 */
enum { RTB_SCHEME_NAME = 0, RTB_SCHEME_RESULT_FILE = 1, RTB_SCHEME_LOG_FILE = 2, RTB_SCHEME_COMMENT = 3 };
typedef struct rtb_scheme rtb_scheme;
/* The <beam> element (scheme.cpp:684-850). */
typedef struct rtb_scheme_beam {
    int32_t type;          /* RTB_BEAM_* */
    int32_t shape;         /* RTB_CIRCLE / RTB_RECTANGLE */
    int32_t profile;       /* RTB_PROFILE_* */
    int32_t range_distr;   /* RTB_RANGE_* */
    double params[6];      /* N, R_in, R_out [, ratio] [, angle or fwhm] */
    int32_t n_params;
    int32_t reserved;
    double center[3];
    uint64_t n_lambda;     /* 0: not a composite beam */
} rtb_scheme_beam;
/* Load a scheme file.  On failure returns RTB_BAD_VALUE (RTB_BAD_ALLOC) and,
 * when scheme_error is not NULL, the Scheme::SchemeError the reference throws
 * (scheme.h:25-27: 0 FileOpenFailure, 1 ParseFailure, 3 BadAttrValue, ...). */
RTB_API int rtb_scheme_load(const char* path, rtb_scheme** scheme, int* scheme_error);
/* The surfaces as rtb_surface (valid until rtb_scheme_free; tables included). */
RTB_API int rtb_scheme_surfaces(const rtb_scheme* scheme, const rtb_surface** surfaces, size_t* n);
/* RTB_SCHEME_NAME, _RESULT_FILE, _LOG_FILE, or RTB_SCHEME_COMMENT + k for
 * surface k's comment; NULL if out of range. */
RTB_API const char* rtb_scheme_text(const rtb_scheme* scheme, int which);
RTB_API int rtb_scheme_get_beam(const rtb_scheme* scheme, rtb_scheme_beam* beam);
/* Wavelength ranges, n_rows rows of row_len numbers: w1 w2 and, for a range
 * file, one order per grating in scheme order (scheme.cpp:1026-1032). */
RTB_API int rtb_scheme_ranges(const rtb_scheme* scheme, const double** rows, size_t* n_rows, size_t* row_len);
RTB_API void rtb_scheme_free(rtb_scheme* scheme);

/* ---- throughput curves (Scheme::ComputeQE, scheme.cpp:1123-1338) ---------- */
/* One surface of ComputeQE's list: a non-AUX surface of type MIRROR, LENS,
 * GRATING or DETECTOR, in document order, with its qe_curve (a number, or a
 * two-column table file).  ComputeQE builds every such surface but a grating
 * as a plain mirror (scheme.cpp:1187-1189), so a DETECTOR's curve counts. */
typedef struct rtb_qe_surface {
    int32_t type;          /* RTB_MIRROR, RTB_LENS, RTB_GRATING or RTB_DETECTOR */
    int32_t reserved;
    rtb_table qe;          /* qe_curve; n == 1 for a single value */
    int64_t order;         /* gratings: the order attribute (used with one range) */
    double gr_const;       /* the const attribute */
    double alpha_deg, gamma_deg, blaze_deg;  /* alpha, gamma, blaze_angle, degrees */
    double rule_start, rule_stop;            /* rule_params: default 0 1; one value v: 0 v */
} rtb_qe_surface;
/* The QE surfaces of a loaded scheme (valid until rtb_scheme_free).  Returns
 * RTB_BAD_VALUE with the SchemeError where ComputeQE fails on them: a missing
 * type, qe_curve or grating attribute (1 ParseFailure), a qe_curve value <= 0,
 * an unreadable table or rule_params whose start >= stop after clamping to
 * [0, 1] (3 BadAttrValue), no QE surface (8 NoSurfaceDesc). */
RTB_API int rtb_scheme_qe_surfaces(const rtb_scheme* scheme, const rtb_qe_surface** surfaces, size_t* n,
                                   int* scheme_error);
/* ComputeQE's curves (scheme.cpp:1249-1316) for n_rows wavelength ranges
 * (rows of row_len numbers, as rtb_scheme_ranges gives them) of n_lambda >= 2
 * wavelengths each, in one launch: lambda[r*n_lambda + i] = w1 +
 * (w2 - w1)/(n_lambda - 1)*i, and qe[r*n_lambda + i] the product, surface after
 * surface, of QE(lambda) (surface_QE) and, for a grating, of its energy in
 * |order| (grating_energy_distr; angles converted as Grating::SetRuleParams
 * does, surface.cpp:595-611).  With more than one range, grating g takes its
 * order from column 2 + g.  Host arrays of n_rows*n_lambda doubles;
 * synchronous.  RTB_OUT_OF_RANGE: a wavelength outside a QE table. */
RTB_API int rtb_qe_curves(const rtb_qe_surface* surfaces, size_t n_surfaces, const double* rows, size_t n_rows,
                          size_t row_len, size_t n_lambda, double* lambda, double* qe);
/* Write curves as ComputeQE writes its QE file (scheme.cpp:1318-1334): one
 * block per range, {size_t n_lambda; double lambda[n_lambda]; double
 * qe[n_lambda]}.  ccd_frame reads one block per ray-tracing file. */
RTB_API int rtb_save_qe(const char* path, size_t n_rows, size_t n_lambda, const double* lambda, const double* qe);

/* ---- reductions of a trace's wavelengths (efficiency/losses_comp.cpp, tools/print_lambda.cpp) ---- */
/* losses_comp's per-wavelength transmission of one result (losses_comp.cpp:
 * 60-90) from the device array lambda of n rays, good rays first (the .dat
 * order): with nl = n / n_lambda, ll[i] is the (i*nl)-th smallest of all n
 * wavelengths and ratio[i] the number of good rays equal to ll[i] among the
 * next nl of the sorted good wavelengths (from where the previous count
 * ended), divided by nl.  The reference reads past the good rays when that
 * window runs over their end; here it stops there.  ll and ratio: host arrays
 * of n_lambda.  Synchronous. */
RTB_API int rtb_loss_ratios(const double* lambda, uint64_t n, uint64_t n_good, uint64_t n_lambda, double* ll,
                            double* ratio, void* stream);
/* print_lambda's list (print_lambda.cpp:36-71): the distinct wavelengths of the
 * good rays lambda[0, n_good) (device) in order of first occurrence, at most
 * max_out of them, into out (host); *n_out their number.  Synchronous. */
RTB_API int rtb_unique_lambdas(const double* lambda, uint64_t n_good, uint64_t max_out, double* out,
                               uint64_t* n_out, void* stream);

/* ---- result files ---------------------------------------------------------- */
/* Write beam [first, first+n) of the device arrays `rays` as a .dat file
 * (Beam::Save, common-lib/beam.cpp:636-715): size_t n, n_good, n_lambda, then
 * X Y Z cX cY cZ lambda of the good rays, then of the lost rays, in the
 * reference's order: order (device) as rtb_reference_order fills it
 * (order[first + k] is the beam-local index of the ray at position k;
 * positions [0, n_good) are the good rays).  Synchronous. */
RTB_API int rtb_save_dat(const char* path, const rtb_rays* rays, const uint32_t* order, uint64_t first, uint64_t n,
                         uint64_t n_good, uint64_t n_lambda, void* stream);
/* Header of a .dat file. */
RTB_API int rtb_read_dat_header(const char* path, uint64_t* n, uint64_t* n_good, uint64_t* n_lambda);
/* Read a .dat file into host arrays of host_rays->n rays (flag, if given,
 * becomes 1 for the first n_good rays and 0 after); a NULL array is skipped. */
RTB_API int rtb_read_dat(const char* path, const rtb_rays* host_rays);
/* Write an image (host, xdim x ydim doubles, row-major, x fastest) as a FITS
 * file with BITPIX -64, as ccd_frame writes its image (ccd/ccd_frame.cpp:
 * 263-314), plus n_keys string keywords (RT_LIST, QE_FILE, SPECFILE, CCDINFO in
 * the reference). */
RTB_API int rtb_write_fits(const char* path, const double* image, uint64_t xdim, uint64_t ydim,
                           const char* const* keys, const char* const* values, size_t n_keys);

/* =========================================================================
 * 4. Adjoint: gradients of the CCD-plane positions with respect to scheme
 *    parameters (no counterpart in the reference).  A forward/backward pair
 *    of the shape a torch.autograd.Function wraps: forward(theta) -> X, Y per
 *    ray; backward(dL/dX, dL/dY) -> dL/dtheta.  The forward is the plain FP64
 *    engine (the same bits as rtb_trace's RTB_FP64 fused engine) and keeps
 *    each ray's state at every surface boundary; the backward recomputes one
 *    surface at a time from those checkpoints, last to first, and carries the
 *    adjoint of the ray state back through it.  Root iterations are
 *    differentiated by the implicit-function theorem at the returned point.
 *    Lost rays carry no gradient (flags are not differentiable).
 * ========================================================================= */
enum {
    RTB_PARAM_CURVATURE = 0,      /* params[0], c (1/mm) */
    RTB_PARAM_CONIC = 1,          /* params[1], conic constant k */
    RTB_PARAM_POLY = 2,           /* params[3 + index], polynomial coefficient a_(index+1) of r^(2 index + 2) */
    RTB_PARAM_TORIC_CR = 3,       /* the toric's cR, params[3 + N] */
    RTB_PARAM_DISTANCE = 4,       /* distance[index], mm */
    RTB_PARAM_ANGLE = 5,          /* angles_deg[index], degrees (about y, x, z) */
    RTB_PARAM_GROOVE_DENSITY = 6  /* grating lines per mm: gr_const = 1000 / value */
};
/* One differentiable scheme parameter: field `kind` (index `index`) of
 * surface `surface`.  A parameter whose change would switch the surface's
 * algorithm (the curvature of a conic at c = 0, the conic constant of a
 * paraboloid, k = -1) is rejected with RTB_BAD_VALUE. */
typedef struct rtb_param {
    int32_t surface;
    int32_t kind;
    int32_t index;
    int32_t reserved;
} rtb_param;
#define RTB_ADJ_MAX_PARAMS 64
typedef struct rtb_adjoint rtb_adjoint;

/* Prepare on the current device: copies of the scheme (tables included), the
 * parameter list, the beam table, and room for n_rays rays' checkpoints
 * (48 bytes x n_surfaces per ray), wavelengths and outputs. */
RTB_API int rtb_adjoint_create(const rtb_surface* surfaces, size_t n_surfaces, const rtb_param* params,
                               size_t n_params, const rtb_beam* beams, size_t n_beams, uint64_t n_rays,
                               uint32_t fixes, rtb_adjoint** ctx);
/* The parameters' values in the scheme given to rtb_adjoint_create (host, n_params). */
RTB_API int rtb_adjoint_theta(const rtb_adjoint* ctx, double* theta);
/* Trace `rays` (device, n_rays, not modified) through the scheme with the
 * parameters set to theta (host, n_params; NULL: the create-time values).
 * X, Y (device, may be NULL) receive the CCD-plane positions and flag
 * (device, may be NULL) 1 for rays that reach the end.  Synchronous. */
RTB_API int rtb_adjoint_forward(rtb_adjoint* ctx, const double* theta, const rtb_rays* rays, double* X, double* Y,
                                char* flag, rtb_trace_stats* stats, void* stream);
/* grad[j] = sum over rays of gX * dX/dtheta_j + gY * dY/dtheta_j for the last
 * forward (gX, gY device, n_rays; grad host, n_params).  Deterministic.  One
 * reverse sweep per ray through the surfaces, each surface recomputed from its
 * checkpoint; with the environment variable RTB_ADJOINT_BACKWARD=passes, the
 * same gradient (to rounding) by forward-mode dual-number passes. */
RTB_API int rtb_adjoint_backward(rtb_adjoint* ctx, const double* gX, const double* gY, double* grad, void* stream);
/* Forward-mode sensitivities of the last forward along dtheta (host, n_params):
 * dX, dY (device, n_rays) = sum_j dtheta_j dX/dtheta_j (0 for lost rays). */
RTB_API int rtb_adjoint_jvp(rtb_adjoint* ctx, const double* dtheta, double* dX, double* dY, void* stream);
/* The spot merit of the last forward: for every wavelength of every beam
 * (group g = beam b, wavelength index j; rays first_ray + j + m * n_lambda)
 * with good rays, RMS spot radius + weight * (centroid x - target_x[g])^2,
 * summed; *merit (host) receives it and gX, gY (device, n_rays, may be
 * NULL) its derivatives with respect to each ray's X and Y, ready for
 * rtb_adjoint_backward.  target_x: host, one value per group, beams in
 * order.  Deterministic. */
RTB_API int rtb_adjoint_spot_merit(rtb_adjoint* ctx, const double* target_x, double weight, double* merit,
                                   double* gX, double* gY, void* stream);
/* The spectral-resolution merit of the last forward: along the dispersion
 * direction u = (ux, uy) on the CCD (normalised here), each group's spot has a
 * centroid p_g and an RMS width s_g; for every pair of neighbouring
 * wavelengths g, g+1 of a beam (both with good rays) the width of a resolution
 * element in wavelength over its mean wavelength,
 *   (s_g + s_g+1) / 2 * |lambda_g+1 - lambda_g| / |p_g+1 - p_g| / ((lambda_g + lambda_g+1) / 2),
 * is summed: the sum of the inverse resolving powers.  lambda: host, the
 * wavelength of each group (beams in order).  *merit, gX, gY as in
 * rtb_adjoint_spot_merit.  RTB_BAD_VALUE for a zero direction, a wavelength
 * that is not positive, or two neighbouring spots with one centroid.  No
 * counterpart in the reference.  Deterministic. */
RTB_API int rtb_adjoint_resolution_merit(rtb_adjoint* ctx, const double* lambda, double ux, double uy, double* merit,
                                         double* gX, double* gY, void* stream);
RTB_API int rtb_adjoint_destroy(rtb_adjoint* ctx);
/* Compile the adjoint's reverse sweep for this scheme's structure ahead of
 * rtb_adjoint_create (which compiles it otherwise, once per structure and
 * process, and launches it from rtb_adjoint_backward; RTB_SPECIALIZE=0 keeps
 * the generic kernel); needs no device.  One kernel serves every parameter
 * value of the structure.  RTB_OK when compiled; RTB_FAILED with the reason
 * in note (may be NULL) when NVRTC is unavailable or fails.  No counterpart
 * in the reference. */
RTB_API int rtb_adjoint_specialize(const rtb_surface* surfaces, size_t n_surfaces, uint32_t fixes, char* note,
                                   size_t note_len);

#ifdef __cplusplus
}
#endif

#endif /* RTB_H */
