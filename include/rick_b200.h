/*
 * rick_b200.h -- C ABI of librick_b200.so, a B200 (sm_100a) implementation of
 * RICK's imaging hot path: convolutional w-stacking gridding, per-w-plane 2-D
 * inverse FFT, and the w-term phase correction summed into the dirty image.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements, ABI-identical to the reference's C prototypes:
 *       wstack            replaces w-stacking.h:39-57  (CPU/CUDA wstack)
 *       phase_correction  replaces w-stacking.h:70-83
 *     plus rick_fft_planes, which does the arithmetic of fftw_data
 *     (fourier_transform.c:13-93) on explicit buffers.  They take host
 *     pointers, accumulate into the output (the CPU path's semantics,
 *     w-stacking.cu:530-532 and phase_correction.cu:233-235) and return void,
 *     like the originals; rick_last_status() reports the outcome.  The
 *     gridding kernel and PHASE_ON, compile-time macros in the reference
 *     (Makefile:56-70), are run-time settings here: rick_set_kernel(),
 *     rick_set_phase_on(), or the RICK_KERNEL / RICK_PHASE_ON environment
 *     variables read on first use.
 *
 *  2. A status-returning plan API for device-resident pipelines: rows live in
 *     HBM, the binned rows, the w-plane cube and cuFFT plans stay allocated
 *     across calls, and every call is asynchronous on the caller's stream.
 *
 * All sizes are plain C types; no CUDA or torch type appears in a signature
 * (streams are passed as void*, meaning cudaStream_t; NULL is the legacy
 * default stream).  Status codes keep errcodes.h:2-6 and add new ones.
 */
#ifndef RICK_B200_H
#define RICK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define RICK_OK                       0
#define RICK_ERR_NO_THREADS_SUPPORT   1   /* errcodes.h:2 */
#define RICK_ERR_IN_PARAMFILE         2   /* errcodes.h:3 */
#define RICK_ERR_NOT_ENOUGH_MEM       3   /* errcodes.h:4 NOT_ENOUGH_MEM_STACKING */
#define RICK_ERR_REDUCE               4   /* errcodes.h:5 */
#define RICK_ERR_INVALID_ARG         16
#define RICK_ERR_CUDA                17
#define RICK_ERR_CUFFT               18
#define RICK_ERR_IO                  19
#define RICK_ERR_UNSUPPORTED         20
#define RICK_ERR_BUDGET              21   /* serving: job does not fit the HBM budget */
#define RICK_ERR_CANCELLED           22
#define RICK_ERR_NO_ACCELERATORS_FOUND 255 /* errcodes.h:6 */

/* ---- gridding kernels (Makefile:63-70 macros) and precision forms -------- */
#define RICK_KERNEL_GAUSS               0  /* -DGAUSS */
#define RICK_KERNEL_GAUSS_HI_PRECISION  1  /* -DGAUSS_HI_PRECISION */
#define RICK_KERNEL_KAISER_BESSEL       2  /* -DKAISERBESSEL (the Makefile default) */

#define RICK_PREC_FP64   0  /* "plain": FP64 grid and Z2Z FFT */
#define RICK_PREC_MIXED  1  /* FP32 grid with FP64 tile sums, C2C FFT, FP64 w-phase */

/* ---- 1. drop-in entry points -------------------------------------------- */

/* w-stacking.h:39-57.  Grids num_points rows onto the w-stacked cube
 * grid[2*num_w_planes*grid_size_y*grid_size_x] (interleaved re,im; index
 * 2*(j + k*grid_size_x + w*grid_size_x*grid_size_y)) and ADDS to it.
 * uu,vv,ww are normalised to [0,1]; dx = 1/grid_size_x, dw = 1/num_w_planes
 * (init.c:11-12).  vis_* hold num_points*freq_per_chan*polarizations floats
 * [row][chan][pol]; weight holds num_points*polarizations [row][pol].
 * Rows whose w-plane index falls outside [0,num_w_planes) are skipped
 * (the reference writes them out of bounds).  num_threads is unused;
 * rank selects device rank % device_count (w-stacking.cu:279-281). */
void wstack(int num_w_planes, unsigned int num_points, unsigned int freq_per_chan,
            unsigned int polarizations, double *uu, double *vv, double *ww, float *vis_real,
            float *vis_img, float *weight, double dx, double dw, int w_support,
            int grid_size_x, int grid_size_y, double *grid, int num_threads, int rank);

/* w-stacking.h:70-83.  image_{real,imag}[yaxis*xaxis] += sum over planes of
 * gridss * exp(2*pi*i*wterm*(sqrt(1-l^2-m^2)-1)) * dwnorm * sqrt(1-l^2-m^2)
 * (phase_correction.cu:191-250), or the plain plane sum when PHASE_ON is off
 * or num_w_planes == 1.  gridss is a host cube laid out like wstack's grid. */
void phase_correction(double *gridss, double *image_real, double *image_imag, int xaxis,
                      int yaxis, int num_w_planes, int xaxistot, int yaxistot,
                      double resolution, double wmin, double wmax, int num_threads, int rank);

/* The arithmetic of fftw_data (fourier_transform.c:13-93): for every w-plane,
 * gridss = FFTW_BACKWARD(grid) / (grid_size_x*grid_size_y).  Host buffers,
 * may alias.  Returns a status. */
int rick_fft_planes(const double *grid, double *gridss, int num_w_planes, int grid_size_x,
                    int grid_size_y);

/* Settings for the drop-ins (compile-time macros in the reference). */
int rick_set_kernel(int kernel);       /* RICK_KERNEL_*; default KAISER_BESSEL */
int rick_set_phase_on(int on);         /* PHASE_ON; default on */
int rick_set_device(int device);       /* overrides rank % device_count */
int rick_last_status(void);            /* status of this thread's last drop-in call */
/* Drop-in resource accounting (no counterpart in the reference): plans the
 * drop-ins have created and device allocations of their row buffers, so far
 * in this process.  The cached plan of a device serves every drop-in call on
 * the same cube geometry, so a repeated wstack -> rick_fft_planes ->
 * phase_correction sequence creates and allocates nothing after its first
 * round. */
int rick_dropin_counters(uint64_t *plans_created, uint64_t *row_allocations);
/* Frees what the drop-ins keep between calls (the cached plans, row and image
 * buffers of every device); the next drop-in call starts afresh.  No
 * counterpart in the reference, whose wstack and phase_correction allocate
 * and free their device memory on every call (w-stacking.cu:316-331, 420-429;
 * phase_correction.cu:137-179). */
int rick_dropin_release(void);
const char *rick_status_string(int status);
const char *rick_last_error_message(void); /* detail of this thread's last failure */

/* ---- 2. plan API (device-resident) -------------------------------------- */

typedef struct rick_plan rick_plan;

typedef struct rick_plan_desc {
  int grid_size_x;        /* Nx */
  int grid_size_y;        /* Ny */
  int num_w_planes;       /* Nw */
  int w_support;          /* odd, 3..15 */
  int kernel;             /* RICK_KERNEL_* */
  int precision;          /* RICK_PREC_* */
  int phase_on;           /* PHASE_ON */
  int device;             /* CUDA device ordinal, -1 = current */
  uint64_t max_rows;      /* capacity: rows per call */
  uint32_t freq_per_chan; /* channels per row */
  uint32_t polarizations; /* polarisations per row (1, 2 or 4 vectorise) */
  /* w-plane shard: the plan holds planes w_first .. w_first+w_count-1 of the
   * num_w_planes-plane cube (0, 0: all).  Rows are assigned to planes with the
   * whole cube's dw; rows of other planes are skipped (rows_other_shard); the
   * image is this shard's part of the plane sum (the w-correction uses the
   * global plane index), so the shards' images add up to the whole image. */
  int w_first;
  int w_count;
  /* NORMALIZE_UVW (gridding.c:21-83): every gridding call first normalises the
   * rows' u, v, w in place on the device (the rows passed to rick_plan_grid /
   * rick_plan_image are rewritten, as the reference rewrites its data arrays;
   * rick_plan_image_host rewrites only its device copies). */
  int normalize_uvw;
} rick_plan_desc;

typedef struct rick_plan_stats {
  uint64_t rows_in;        /* rows passed to the last gridding call */
  uint64_t rows_gridded;   /* rows that reached the grid */
  uint64_t rows_dropped;   /* rows outside the cube or the one-rank sector */
  uint64_t records;        /* binned row records (rows touching k tiles count k) */
  uint64_t work_items;     /* gridder work items (tile chunks) */
  uint64_t device_bytes;   /* HBM held by the plan */
  uint64_t fft_rows;       /* (plane, row) pairs the last rick_plan_image transformed on its
                              sparse path (rows the gridder touched); 0 after the dense path */
  uint64_t rows_other_shard; /* rows of planes outside the plan's w-plane shard */
} rick_plan_stats;

/* Row selection applied by the gridding calls. */
#define RICK_ROWS_ALL      0  /* wstack semantics: grid every row given */
#define RICK_ROWS_SECTOR0  1  /* gridding() semantics for one rank: the sector-0 rows of
                                 gridding.c:149-188 (incl. the v-halo rule) */

int rick_plan_create(rick_plan **plan, const rick_plan_desc *desc);
int rick_plan_destroy(rick_plan *plan);
/* Bytes of HBM a plan with this description would hold (for admission).  On
 * power-of-two grids (the sparse-aware FFT of rick_plan_image) this excludes the
 * cuFFT work area, which the stage call rick_plan_fft allocates on first use. */
int rick_plan_footprint(const rick_plan_desc *desc, uint64_t *bytes);

/* Grid device-resident rows into the plan's cube (overwrites the cube). */
int rick_plan_grid(rick_plan *plan, uint64_t nrows, const double *uu, const double *vv,
                   const double *ww, const float *weight, const float *vis_real,
                   const float *vis_img, int row_selection, void *stream);
/* In-place inverse FFT of every plane of the cube (FFTW_BACKWARD sign); the
 * 1/(Nx*Ny) scale is carried and applied by rick_plan_phase / export. */
int rick_plan_fft(rick_plan *plan, void *stream);
/* image = (accumulate ? image : 0) + w-corrected plane sum; device pointers,
 * Ny*Nx doubles each.  resolution = 1/max(|uvmin|,|uvmax|) (gridding_cpu.c:78). */
int rick_plan_phase(rick_plan *plan, double resolution, double wmin, double wmax,
                    double *image_real, double *image_imag, int accumulate, void *stream);
/* grid + fft + phase in one call (stream-ordered, no host synchronisation). */
int rick_plan_image(rick_plan *plan, uint64_t nrows, const double *uu, const double *vv,
                    const double *ww, const float *weight, const float *vis_real,
                    const float *vis_img, int row_selection, double resolution, double wmin,
                    double wmax, double *image_real, double *image_imag, void *stream);
/* The same with HOST buffers: rows are copied to HBM (pinned staging,
 * overlapped with binning), the image is copied back; synchronous. */
int rick_plan_image_host(rick_plan *plan, uint64_t nrows, const double *uu, const double *vv,
                         const double *ww, const float *weight, const float *vis_real,
                         const float *vis_img, int row_selection, double resolution,
                         double wmin, double wmax, double *image_real, double *image_imag);
/* Copy the cube out as FP64 interleaved (wstack layout), scaled to the
 * FFTW-normalised values when it has been transformed.  dst may be host or
 * device memory (is_host). Adds into dst when accumulate != 0 (device dst only). */
/* Streaming ingest: the same imaging as rick_plan_image_host for a dataset whose
 * samples arrive in slices of rows (read from disk while earlier slices copy
 * and bin).  begin takes the host arrays of every row's u, v, w and weights
 * and runs the position pass; samples takes the host vis_real / vis_img of rows
 * row0 .. row0+nrows-1, in increasing row order, copies them asynchronously
 * and bins them -- the buffers of one call may be reused once the next call
 * has returned (pinned buffers make the copies overlap); end grids, transforms
 * and corrects, and writes the host image (synchronises).  A begin while an
 * ingest is unfinished abandons it. */
int rick_plan_ingest_begin(rick_plan *plan, uint64_t nrows, const double *uu, const double *vv,
                           const double *ww, const float *weight, int row_selection);
int rick_plan_ingest_samples(rick_plan *plan, uint64_t row0, uint64_t nrows,
                             const float *vis_real, const float *vis_img);
int rick_plan_ingest_end(rick_plan *plan, double resolution, double wmin, double wmax,
                         double *image_real, double *image_imag);

int rick_plan_export_cube(rick_plan *plan, double *dst, int dst_is_host, void *stream);
/* Load an FP64 interleaved cube (host or device) into the plan, marked as
 * already transformed and normalised (phase_correction's input). */
int rick_plan_import_cube(rick_plan *plan, const double *src, int src_is_host, void *stream);
int rick_plan_get_stats(rick_plan *plan, rick_plan_stats *stats); /* synchronises */

/* Stage timers (the counterpart of the reference's timing_wt stage times,
 * timing.h:60-76): when enabled, every plan call records CUDA events around
 * its stages on the caller's stream; rick_plan_stage_ms reports the last call's
 * milliseconds per stage (synchronises) in the order
 *   0 bin_count (histogram + scans), 1 bin_scatter (row sums + records),
 *   2 cube_zero, 3 grid (tiled gridder), 4 fft, 5 phase (w-correction + sum);
 * a stage that did not run in the last call reports -1. */
#define RICK_NUM_STAGES 6
int rick_plan_set_timing(rick_plan *plan, int on);
int rick_plan_stage_ms(rick_plan *plan, float *ms, int n);

/* ---- 3. gridding without device allocation ------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory at run time -- real-time pipelines that reserve all GPU memory at
 * start-up and may not grow it inside their streaming loop, or host frameworks
 * that own the device memory pool -- this grids device-resident rows
 * (wstack's arguments, as device pointers, all rows gridded) into the caller's
 * device cube grid[2*Nw*Ny*Nx] (overwritten) without calling cudaMalloc: its
 * scratch is one static __device__ array of 32 MiB that every GPU loading the
 * library holds until exit.  A job whose scratch does not fit is rejected with
 * RICK_ERR_INVALID_ARG (rick_wstack_noalloc_capacity gives the row limit for a
 * geometry).  All calls share that array and it keeps the last call's
 * contents; calls whose GPU work overlaps race on it.  The first call on a
 * device sets the device up (looks up the arrays' device addresses and fills
 * a second static array with the kernel tables of every kernel and support,
 * synchronously), so make it before any stream capture: a first call on a
 * capturing stream is refused with RICK_ERR_INVALID_ARG.  Later calls copy
 * nothing from the host.  Asynchronous on `stream`. */
int rick_wstack_noalloc(int num_w_planes, uint64_t num_points, uint32_t freq_per_chan,
                        uint32_t polarizations, const double *uu, const double *vv,
                        const double *ww, const float *vis_real, const float *vis_img,
                        const float *weight, double dx, double dw, int w_support, int kernel,
                        int grid_size_x, int grid_size_y, double *grid, void *stream);
int rick_wstack_noalloc_capacity(int num_w_planes, int grid_size_x, int grid_size_y,
                                 uint64_t *max_rows);

/* NORMALIZE_UVW of gridding.c:21-83 on device rows, in place, asynchronous on
 * `stream`: u, v -> (x + maxg) / (2 maxg) with maxg = 1.001 * the largest
 * |extremum| of u and v, w -> (w - min w) / (max w - min w), the extrema
 * taken over the rows with minima starting at 1e20 and maxima at 0 as in the
 * reference.  scratch: device memory of RICK_NORMALIZE_SCRATCH bytes, 8-byte
 * aligned; when the call has run, its first 7 doubles are min u, min v, min w,
 * max u, max v, max w and maxg. */
#define RICK_NORMALIZE_SCRATCH 128
int rick_normalize_uvw(uint64_t nrows, double *uu, double *vv, double *ww, void *scratch,
                       void *stream);

/* ---- 4. Batched imaging -------------------------------------------------
 * No counterpart in the reference (one rank images one dataset per run).  Many
 * independent imaging jobs of uneven sizes -- each one rick_plan_image call:
 * gridding, per-plane inverse FFT, w-correction and plane sum -- run as one
 * launch per stage over all jobs, the stage sequence captured once in a CUDA
 * graph.  Job inputs and images are device pointers that must stay valid
 * while the batch exists; every run recomputes every image from the rows
 * (images are overwritten).  Grid axes are powers of two in [64, 4096]. */
#define RICK_BATCH_MAX_GRID 4096

typedef struct rick_job_desc {
  int grid_size_x, grid_size_y, num_w_planes, w_support, kernel;
  uint64_t num_rows;
  uint32_t freq_per_chan, polarizations;
  int row_selection;   /* RICK_ROWS_ALL or RICK_ROWS_SECTOR0 */
  int phase_on;        /* PHASE_ON of phase_correction.cu */
  double resolution, wmin, wmax;
  const double *uu, *vv, *ww;            /* device [num_rows], normalised */
  const float *weight;                   /* device [num_rows * polarizations] */
  const float *vis_real, *vis_img;       /* device [num_rows * freq_per_chan * polarizations] */
  double *image_real, *image_imag;       /* device [grid_size_y * grid_size_x] */
} rick_job_desc;

/* Schedule knobs of a batch: gridder records per work item, gridder blocks per
 * SM, and the column pass's form: planes_in_flight 0 keeps each pixel's running
 * sum and w-step in tensor memory (one plane per iteration); 1 or 2 keep them
 * in registers with that many planes per iteration (2: mixed form only). */
typedef struct rick_batch_tuning {
  uint32_t max_chunk;
  int grid_blocks_per_sm;
  int planes_in_flight;
} rick_batch_tuning;

typedef struct rick_batch rick_batch;

/* HBM the batch holds (cubes, column-blocked planes, records, tables). */
int rick_batch_footprint(const rick_job_desc *jobs, int njobs, int precision, uint64_t *bytes);
/* Creates the batch on `device` (precision RICK_PREC_*).  tuning == NULL runs
 * the autotuner (times candidate schedules on the batch itself, synchronises,
 * writes the images; results cached per batch shape for the process). */
int rick_batch_create(rick_batch **batch, const rick_job_desc *jobs, int njobs, int precision,
                      int device, const rick_batch_tuning *tuning);
/* One graph launch on `stream` (a cudaStream_t); asynchronous. */
int rick_batch_run(rick_batch *batch, void *stream);
int rick_batch_get_tuning(rick_batch *batch, rick_batch_tuning *tuning);
/* Kernel launches one run replays from the graph (all jobs together). */
int rick_batch_kernels_per_run(rick_batch *batch, uint32_t *kernels);
/* Totals over all jobs of the last run (synchronises). */
int rick_batch_get_stats(rick_batch *batch, rick_plan_stats *stats);
int rick_batch_destroy(rick_batch *batch);

/* ---- 5. Served imaging ---------------------------------------------------
 * No counterpart in the reference.  A request loop with continuous batching:
 * jobs are submitted from any thread as they arrive; a scheduler thread admits
 * waiting jobs (oldest first) while their HBM footprint fits the budget,
 * launches them as one batch on a free stream, and keeps admitting while
 * earlier batches run, so batches overlap on the device.  Job rows and images
 * are device pointers owned by the caller and must stay valid until the job's
 * wait returns.  Each job's image is the same as imaging it alone (within the
 * precision's tolerance: tiles split over work items add in any order). */
typedef struct rick_server rick_server;

typedef struct rick_server_desc {
  int device;
  int precision;          /* RICK_PREC_* */
  uint64_t hbm_budget;    /* bytes of working memory the admitted jobs may hold */
  int max_batch_jobs;     /* jobs per launched batch at most */
  int streams;            /* batches on the device at once at most */
  uint64_t solo_vis;      /* jobs with at least this many visibilities run as a batch of their
                             own, beside the small-job batches (0: 5e7) */
} rick_server_desc;

typedef struct rick_job_result {
  int status;
  double queue_ms;        /* submit -> launch */
  double latency_ms;      /* submit -> image complete on the device */
  uint64_t batch_id;
  uint32_t batch_jobs;    /* jobs of the batch it ran in */
} rick_job_result;

typedef struct rick_server_stats {
  uint64_t jobs_submitted, jobs_done, vis_done, batches;
  uint64_t bytes_in_use, peak_bytes, jobs_waiting;
} rick_server_stats;

/* Reserves the whole budget in the server's stream-ordered pool at creation
 * (RICK_ERR_NOT_ENOUGH_MEM if the device cannot hold it). */
int rick_server_create(rick_server **server, const rick_server_desc *desc);
/* Queues one job; RICK_ERR_BUDGET when the job alone exceeds the budget. */
int rick_server_submit(rick_server *server, const rick_job_desc *job, uint64_t *ticket);
/* Waits for the job (timeout_ms < 0: no limit; RICK_ERR_CANCELLED on timeout)
 * and returns its status; the ticket is released. */
int rick_server_wait(rick_server *server, uint64_t ticket, double timeout_ms,
                     rick_job_result *result);
int rick_server_get_stats(rick_server *server, rick_server_stats *stats);
/* Cancels a job still waiting for admission: its wait returns
 * RICK_ERR_CANCELLED.  A job already launched is never interrupted (no kernel
 * is stopped part-way); for it, and for unknown tickets, this returns
 * RICK_ERR_INVALID_ARG and the job completes as usual.  The reference's
 * counterpart is a failed rank ending the run (main.c:6-28, errcodes.h). */
int rick_server_cancel(rick_server *server, uint64_t ticket);
/* Stops admitting jobs: submit returns RICK_ERR_CANCELLED from now on.  With
 * drain != 0 every waiting job still runs; with drain == 0 the waiting jobs
 * are cancelled (their waits return RICK_ERR_CANCELLED) while the launched
 * batches finish.  Does not block. */
int rick_server_shutdown(rick_server *server, int drain);
/* Finishes every submitted (and not cancelled) job, then releases the server. */
int rick_server_destroy(rick_server *server);

/* Page-locked host memory (for the buffers of rick_plan_ingest_samples and
 * rick_plan_image_host, whose copies then run asynchronously). */
int rick_host_alloc(void **ptr, uint64_t bytes);
int rick_host_free(void *ptr);

/* Names of the kernels this library launches, and how many launches it has
 * issued in this process (for launch accounting). */
int rick_kernel_names(const char **names, int max_names);
unsigned long long rick_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* RICK_B200_H */
