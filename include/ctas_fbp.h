/*
 * ctas_fbp.h -- C ABI of the B200 parallel-beam filtered-backprojection path.
 *
 * This is the drop-in boundary for the reconstruction class of ctas
 * (class CTrec, src/common/ct.h:235-298, implemented in src/common/lct.cpp:
 * 487-729).  A handle `ctas_fbp` plays the role of one CTrec object: it holds
 * the sinogram shape, contrast, filter window, angle table and physics
 * coefficient, and owns the device buffers and the CUDA stream.  Every entry
 * point returns an int status (CTAS_OK == 0, negative on error) instead of
 * throwing CtasErr (src/common/common.world.cpp:165-170); the message of the
 * last failure on the calling thread is returned by ctas_fbp_last_error().
 *
 * Array conventions (ctas `Map`, src/common/matrix.world.h:127-129): a
 * sinogram is row-major float32 [n_angles][width] (row = projection), a slice
 * is row-major float32 [rows][cols] (W x W unless an output geometry is set).
 * Host pointers are plain CPU memory (pinned memory is faster); `_dev`
 * variants take CUDA device pointers and a cudaStream_t passed as void*.
 *
 * There is no CPU fallback: without a usable CUDA device the create call
 * fails with CTAS_E_NODEVICE.
 */
#ifndef CTAS_FBP_H
#define CTAS_FBP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------- status codes */
#define CTAS_OK              0
#define CTAS_E_ARG          -1  /* invalid argument: null pointer, bad enum, bad option  */
#define CTAS_E_SHAPE        -2  /* W < 2 or N == 0 (lct.cpp:500-503); shape too large   */
#define CTAS_E_CENTER       -3  /* |center| >= W/2 (lct.cpp:614-616, 651-653)           */
#define CTAS_E_FILTER       -4  /* unknown filter (lct.cpp:83-84); bad Kaiser/Gauss
                                   parameter (ct.h:148-151)                             */
#define CTAS_E_DATA         -5  /* bad absorption data: maximum <= 0
                                   (physical.world.cpp:93-94)                           */
#define CTAS_E_STATE        -6  /* repeat() before sino()                               */
#define CTAS_E_CUDA         -7  /* CUDA runtime error                                   */
#define CTAS_E_NOMEM        -8  /* device or host allocation failed                     */
#define CTAS_E_UNSUPPORTED  -9  /* option combination not supported                     */
#define CTAS_E_NODEVICE    -10  /* no CUDA device                                       */
#define CTAS_E_TIMEOUT     -11  /* a bounded device wait ran out (kernel returned early) */
#define CTAS_E_IO          -12  /* a volume read or write callback failed (ctas_volume.h) */

/* ----------------------------------------------- Contrast::Cntype (physical.world.h:22-27) */
enum { CTAS_ABS = 0, CTAS_REF = 1, CTAS_PHS = 2, CTAS_FLT = 3 };

/* ------------------------------------------------- Filter::Ftype (ct.h:92-132) */
enum {
  CTAS_FILTER_NONE = 0, CTAS_FILTER_RAMP = 1, CTAS_FILTER_BARLETT = 2,
  CTAS_FILTER_WELCH = 3, CTAS_FILTER_PARZEN = 4, CTAS_FILTER_HANN = 5,
  CTAS_FILTER_HAMMING = 6, CTAS_FILTER_BLACKMAN = 7, CTAS_FILTER_LANCKZOS = 8,
  CTAS_FILTER_KAISER = 9, CTAS_FILTER_GAUSS = 10,
  /* extensions, no reference counterpart */
  CTAS_FILTER_SHEPP_LOGAN = 100, /* sin(pi f/2)/(pi f/2), f = |k|/(P/2) */
  CTAS_FILTER_COSINE = 101       /* cos(pi f/2)                         */
};

/* --------------------------------------------------------------- options */
enum {
  CTAS_INTERP_TRUNC = 0,  /* reference rule: sample (int)t, bit-compatible (lct.cpp:711-713) */
  CTAS_INTERP_LINEAR = 1  /* extension: linear interpolation, sample k centred at k+0.5 */
};
enum { CTAS_STORE_F32 = 0, CTAS_STORE_F16 = 1, CTAS_STORE_BF16 = 2 };

/* Do not copy the filtered sinogram back into the caller's host buffer.
 * CTrec::reconstruct/sino filter in place (lct.cpp:655, 605-606); callers
 * that discard the sinogram afterwards (the ct tool, ct.cpp:199-202) may set
 * this to save the device->host copy. */
#define CTAS_FLAG_NO_WRITEBACK 0x1u
/* Round the index expression of the backprojection (lct.cpp:711-712) the way
 * the reference's CPU path rounds it as built: its -ffast-math flag
 * (CMakeLists.txt:10-11) makes GCC fold (1 - sin) - cos into 1 - (sin + cos),
 * even at -O0, so that build computes c + (1 - (sin + cos)) * hp + ...  Without
 * the flag the index follows ct.cl:36-37 as written, c + ((1 - sin) - cos) *
 * hp + ..., which is the reference's OpenCL path (and its CPU path built
 * without -ffast-math).  The two choose a different sample for about one
 * update in 10^3-10^4; each rule is bit-exact against its reference build. */
#define CTAS_FLAG_SHIPPED_INDEX 0x2u
/* Run the staged backprojection kernel with every shared-memory gather
 * bounds-checked (a test aid; violations are reported as CTAS_E_CUDA). */
#define CTAS_FLAG_CHECKED 0x100u
/* Test aid: the staged backprojection kernel leaves its first chunk of
 * projection windows uncopied and waits a short bounded time, so its waits run
 * out; the call reports CTAS_E_TIMEOUT and the device stays usable.  (The
 * timeout path of the kernel: drain, error word, early return.) */
#define CTAS_FLAG_TEST_TIMEOUT 0x200u

typedef struct ctas_fbp_opts {
  uint32_t struct_size;   /* sizeof(ctas_fbp_opts); 0 is treated as "all defaults" */
  int32_t interp;         /* CTAS_INTERP_*                                          */
  int64_t pad;            /* zero-padded FFT length; 0 = reference rule
                             2^ceil(log2(2W-1)) (lct.cpp:490); else a power of two
                             >= W + 1                                              */
  int32_t store;          /* CTAS_STORE_*: precision of the filtered sinogram kept
                             on the device                                         */
  int32_t device;         /* CUDA device ordinal; -1 = current device              */
  const double *angles;   /* NULL: th_i = i*arc/N (lct.cpp:512-517); else n_angles
                             projection angles in radians (extension)             */
  int64_t out_rows;       /* output geometry (extension): out_rows x out_cols pixels of
                             pitch out_pixel (detector pixels), centred like the
                             reference's W x W grid and shifted by (out_shift_row,
                             out_shift_col) output pixels; 0 = W                    */
  int64_t out_cols;
  double out_pixel;       /* 0 = 1; the staged kernel serves pitches <= 1           */
  double out_shift_row;
  double out_shift_col;
  uint32_t flags;         /* CTAS_FLAG_*                                            */
  int32_t chunk_slices;   /* slices per device batch in the stack calls (the host
                             form ramps up to it and down again at the ends);
                             0 = auto                                              */
  int32_t tile;           /* staged backprojection tile id in
                             [0, ctas_fbp_tile_count()); -1 = autotune: the first
                             launch of a shape times candidate tiles on one slice
                             (this synchronises the stream once; do it before any
                             stream capture); with struct_size below this field: -1 */
  int32_t ring_box;       /* half width of the ring-artefact filter applied to every
                             sinogram before filtering (RingFilter::apply,
                             lct.cpp:295-327; the ct tool's -R); 0 = off          */
} ctas_fbp_opts;

typedef struct ctas_fbp ctas_fbp;

/* -------------------------------------------------------------- errors */
/* Message of the last failing call on this thread ("" if none). */
const char *ctas_fbp_last_error(void);
const char *ctas_fbp_version(void);

/* ------------------------------------------------ host-side helpers (no GPU) */
/* Filter::fromName (lct.cpp:70-86): case-insensitive; "" -> RAMP,
 * "BARLETT" -> RAMP; extensions "SHEPP-LOGAN"/"SHEPP_LOGAN", "COSINE". */
int ctas_filter_from_name(const char *name, int32_t *ftype);
/* Filter::name (lct.cpp:93-109); NULL for an unknown type. */
const char *ctas_filter_name(int32_t ftype);
/* Filter::Filter parameter checks (ct.h:144-152). */
int ctas_filter_check(int32_t ftype, float param);
/* _conversion(Filter*) (lct.cpp:236-248): "NAME[:float]". */
int ctas_filter_parse(const char *spec, int32_t *ftype, float *param);
/* Filter::fill (lct.cpp:122-209): `pixels` window values into out. */
int ctas_filter_fill(int32_t ftype, float param, int64_t pixels, float *out);
/* Contrast(const std::string&) (physical.world.cpp:19-27) and Contrast::name. */
int ctas_contrast_from_name(const char *name, int32_t *contrast);
const char *ctas_contrast_name(int32_t contrast);
/* Padded FFT length rule P = 2^ceil(log2(2W-1)) (lct.cpp:490). */
int64_t ctas_fbp_padded_width(int64_t width);
/* arcO / angO (lct.cpp:470-484), radians. */
float ctas_fbp_arc(float anarc, int64_t points);
float ctas_fbp_angle(float anarc, int64_t points);
/* cossins table (lct.cpp:512-517): tab[2i] = sinf(th_i), tab[2i+1] = cosf(th_i). */
int ctas_fbp_angle_table(float arc_deg, int64_t n_angles, float *tab);
/* The CTrec window: Filter::fill(P) * P/W, G[0] = 0 for REF (lct.cpp:505-508). */
int ctas_fbp_window(int64_t width, int32_t contrast, int32_t ftype, float fparam,
                    int64_t pad, float *G);
/* setPhysics coefficient (lct.cpp:558-566), SI units. */
float ctas_fbp_rec_cof(float pixel_size_m, float lambda_m);

/* ------------------------------------------------------------ the handle */
/* CTrec::CTrec(sinoshape, cn, anarc, ft) (lct.cpp:487-526).  opts may be NULL. */
int ctas_fbp_create(ctas_fbp **out, int64_t n_angles, int64_t width,
                    int32_t contrast, int32_t ftype, float fparam, float arc_deg,
                    const ctas_fbp_opts *opts);
/* CTrec::CTrec(CTrec&) (lct.cpp:529-545): same set-up, own work buffers and
 * stream, so clones used from different host threads run concurrently. */
int ctas_fbp_clone(const ctas_fbp *src, ctas_fbp **out);
/* CTrec::~CTrec (lct.cpp:549-555).  NULL is accepted. */
int ctas_fbp_destroy(ctas_fbp *h);
/* CTrec::setPhysics (lct.cpp:558-566), SI units (metres). */
int ctas_fbp_set_physics(ctas_fbp *h, float pixel_size_m, float lambda_m);
/* CTrec::recShape (ct.h:272-274): (W - 2k) x W with k = ceil(abs(center)),
 * where abs is the C library's int abs() (the only one in scope in ct.h): the
 * centre is truncated toward zero first, so k = |(int)center|. */
/* (reference grid; with an output geometry the slice is out_rows x out_cols) */
int ctas_fbp_rec_shape(const ctas_fbp *h, float center, int64_t *rows, int64_t *cols);
/* Output slice shape of this handle (W x W unless an output geometry is set). */
int ctas_fbp_out_shape(const ctas_fbp *h, int64_t *rows, int64_t *cols);
/* Sinogram shape of this handle (CTrec::ish: projections x detector pixels). */
int ctas_fbp_sino_shape(const ctas_fbp *h, int64_t *n_angles, int64_t *width);

/* CTrec::sino (lct.cpp:600-609): filter `sino_inout` (n_angles x width) and
 * keep it on the device for ctas_fbp_repeat; the filtered sinogram is written
 * back into sino_inout unless CTAS_FLAG_NO_WRITEBACK. Synchronous. */
int ctas_fbp_sino(ctas_fbp *h, float *sino_inout);
/* CTrec::repeat (lct.cpp:612-646): backproject the kept sinogram with another
 * centre.  Synchronous. */
int ctas_fbp_repeat(ctas_fbp *h, float *slice_out, float center);
/* CTrec::reconstruct (lct.cpp:649-685): filter (in place, see above) and
 * backproject into slice_out.  Synchronous. */
int ctas_fbp_reconstruct(ctas_fbp *h, float *sino_inout, float *slice_out,
                         float center);

/* Device-pointer forms, asynchronous on `stream` (a cudaStream_t; NULL = the
 * legacy default stream).  Errors detected on the device (bad absorption
 * data) are reported by the next ctas_fbp_synchronize. */
int ctas_fbp_sino_dev(ctas_fbp *h, const float *sino_dev, float *filtered_dev,
                      void *stream);
int ctas_fbp_repeat_dev(ctas_fbp *h, float *slice_dev, float center, void *stream);
/* Extension of CTrec::repeat (lct.cpp:610-647): backprojects the sinogram of
 * the last sino() call at n centres (host array, each |c| < W/2) into n
 * consecutive output slices of slices_dev (device), in one launch -- the
 * filter-once / backproject-many loop of the axis search (lct.cpp:865-870).
 * Synchronises `stream` on entry (the centres are staged in a handle-owned
 * device buffer); n <= 65535. */
int ctas_fbp_repeat_multi_dev(ctas_fbp *h, const float *centers, int64_t n,
                              float *slices_dev, void *stream);
int ctas_fbp_reconstruct_dev(ctas_fbp *h, const float *sino_dev, float *slice_dev,
                             float center, void *stream);
int ctas_fbp_synchronize(ctas_fbp *h);

/* A stack of n_slices sinograms of this handle's shape, all with the same
 * centre (the ct tool's slice loop, ct.cpp:170-206).  Host form: pipelined
 * host->device, compute and device->host copies; sinos_inout receives the
 * filtered sinograms unless CTAS_FLAG_NO_WRITEBACK.  Device form: contiguous
 * [n_slices][N][W] input and [n_slices][rows][cols] output. */
int ctas_fbp_reconstruct_stack(ctas_fbp *h, float *sinos_inout, float *slices_out,
                               int64_t n_slices, float center);
int ctas_fbp_reconstruct_stack_dev(ctas_fbp *h, const float *sinos_dev,
                                   float *slices_dev, int64_t n_slices,
                                   float center, void *stream);

/* Which backprojection kernel the last call on this handle used:
 * 0 = none yet, 1 = generic (any angles), 2 = staged fast path (all sines >= 0). */
int ctas_fbp_last_kernel(const ctas_fbp *h);
/* Tile id the staged backprojection kernel used in the last call (-1: none). */
int ctas_fbp_last_tile(const ctas_fbp *h);
/* Number of staged backprojection tile ids (pixel-tile shape x arithmetic
 * variant); valid ids are 0 .. count-1.  Needs no device. */
int ctas_fbp_tile_count(void);
/* Pixel-tile rows x columns and detector-window length (samples fetched per
 * projection) of a staged tile id.  Needs no device. */
int ctas_fbp_tile_shape(int32_t tile, int32_t *rows, int32_t *cols, int32_t *window);
/* Number of CUDA kernels this handle has launched so far. */
int64_t ctas_fbp_kernel_launches(const ctas_fbp *h);

/* Kernel timing (a measurement aid, no reference counterpart).  While enabled,
 * every kernel this handle launches is bracketed by CUDA events recorded on
 * its launch stream.  ctas_fbp_profile_read synchronises, returns the summed
 * device time and launch count of one kind (0 = filter, 1 = backprojection,
 * 2 = other) since the last read, and clears the records of that kind. */
enum { CTAS_KERNEL_FILTER = 0, CTAS_KERNEL_BACKPROJECT = 1, CTAS_KERNEL_OTHER = 2 };
int ctas_fbp_set_profiling(ctas_fbp *h, int enable);
int ctas_fbp_profile_read(ctas_fbp *h, int kind, double *total_ms, int64_t *launches);

/* --------------------------------------------------------- uneven batches
 * Extension (no reference counterpart; the reference reconstructs one
 * sinogram per CTrec call): many sinograms of different widths, projection
 * counts and centres, filtered and backprojected by one filter launch and one
 * persistent backprojection launch, replayed as a CUDA graph.  All sinograms
 * share contrast (PHS, REF or FLT), filter, arc (every sine >= 0) and physics.
 * The device pointers are fixed at create time; put new data in the same
 * buffers and run again.  Create autotunes the tile shape on the batch itself
 * (synchronising) and captures the graph. */
typedef struct ctas_fbp_job {
  int64_t n_angles;
  int64_t width;
  float center;
  const float *sino_dev;  /* n_angles x width, device */
  float *slice_dev;       /* width x width, device */
} ctas_fbp_job;

typedef struct ctas_fbp_batch ctas_fbp_batch;

int ctas_fbp_batch_create(ctas_fbp_batch **out, const ctas_fbp_job *jobs, int64_t n_jobs,
                          int32_t contrast, int32_t ftype, float fparam, float arc_deg,
                          float pixel_size_m, float lambda_m, const ctas_fbp_opts *opts);
/* One graph launch on `stream` (asynchronous). */
int ctas_fbp_batch_run(ctas_fbp_batch *b, void *stream);
/* The same work as a loop of per-sinogram filter + backprojection launches
 * (asynchronous; for comparison, same results). */
int ctas_fbp_batch_run_loop(ctas_fbp_batch *b, void *stream);
/* Waits for the device and reports device-side errors of earlier runs. */
int ctas_fbp_batch_synchronize(ctas_fbp_batch *b);
/* Tile id chosen by the autotuner. */
int ctas_fbp_batch_tile(const ctas_fbp_batch *b);
int ctas_fbp_batch_destroy(ctas_fbp_batch *b);

/* ------------------------------------------------ reconstruction without allocation
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they reconstruct -- code running under a framework that owns
 * every device allocation (a memory pool, a graph-replay runtime that forbids
 * cudaMalloc), acquisition loops with a fixed memory budget, plug-ins that must
 * not touch their host process's allocator: filter + backprojection of one
 * sinogram (sino_dev, n_angles x width) into slice_dev (width x width), both
 * device pointers, with the arguments of ctas_fbp_create / set_physics /
 * reconstruct in one call.  It calls no cudaMalloc, cudaFree or allocating
 * library routine: its scratch (filtered sinogram, FFT tables, angle table) is
 * one fixed 32 MiB array inside the library, which every GPU that loads the
 * library holds until the process exits.  Sizes whose scratch exceeds 32 MiB
 * (n_angles * (width + ~9) * 4 bytes plus the tables; 1800 x 2560 fits) are
 * rejected with CTAS_E_SHAPE; absorption contrast is rejected with
 * CTAS_E_UNSUPPORTED.  The first call on a device looks up the array's device
 * address once for that device.  The call waits for its own work before it
 * returns, so it cannot run on a stream that is being captured: such a stream
 * is refused with CTAS_E_ARG.  All calls in a process share the array, so
 * calls whose GPU work overlapped would race: calls are serialised by a lock,
 * and each returns only after its own work on `stream` has finished, on the
 * error paths too.  The array keeps the previous call's contents; every call
 * clears what must start at zero. */
int ctas_fbp_reconstruct_dev_noalloc(const float *sino_dev, float *slice_dev,
                                     int64_t n_angles, int64_t width, int32_t contrast,
                                     int32_t ftype, float fparam, float arc_deg, int64_t pad,
                                     float center, float pixel_size_m, float lambda_m,
                                     void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CTAS_FBP_H */
