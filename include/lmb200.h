/*
 * lmb200.h -- C ABI of the B200 orientation-matching library (liblmb200.so).
 *
 * The reference LaueMatching has no library interface: its hot path lives
 * inside three executables (src/LaueMatchingCPU.c, src/LaueMatchingGPU.cu,
 * src/LaueMatchingGPUStream.cu) that callers drive through argv and files.
 * Each entry point below replaces one piece of that code path; its comment
 * names the reference lines it replaces.  A binding for ctypes, cgo or any
 * other FFI needs only this header: plain C types, opaque handles, int status.
 *
 * Conventions
 *   - Every call returns LMB_OK (0) or a negative LMB_ERR_* code; the message
 *     of the last failure on the calling thread is in lmb_last_error().
 *   - The caller owns every host buffer; an engine owns its device buffers.
 *   - Calls on one engine are not re-entrant: serialise them per engine.
 *   - Record layout: uint16[1 + 2*S] = {count, x0, y0, x1, y1, ...}, zero
 *     padded, S = MaxNrLaueSpots (LaueMatchingCPU.c:488-495).
 *   - Pixel (x, y) of a row-major image is element y*NrPxX + x
 *     (LaueMatchingCPU.c:676).
 */
#ifndef LMB200_H
#define LMB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMB_OK 0
#define LMB_ERR_INVALID (-1)  /* bad argument or state */
#define LMB_ERR_CUDA (-2)     /* CUDA runtime failure (message has details) */
#define LMB_ERR_OOM (-3)      /* device or pinned host allocation failed */
#define LMB_ERR_OVERFLOW (-4) /* a survivor list exceeded its capacity */
#define LMB_ERR_TIMEOUT (-5)  /* a bounded device wait gave up */

#define LMB_MAX_SLOTS 64 /* images one DB pass can serve */

/* Image pixel types accepted by lmb_image_load. */
#define LMB_F64 0 /* raw float64, the .bin image of the LaueMatchingGPU CLI */
#define LMB_F32 1 /* float32, the TCP wire payload of LaueMatchingGPUStream */
#define LMB_U8 2  /* uint8 frame (values taken as float64, then quantised) */

/* Intensity sources of a compare pass. */
#define LMB_VALUE_U8 0  /* uint8 image x imScale (LaueMatchingCPU.c:668-682) */
#define LMB_VALUE_F64 1 /* float64 image (the DoFwd 1 path, :649-653) */

/* Detector / crystal geometry, all FP64, built by lmb_geometry_init. */
typedef struct lmb_geometry {
  double recip[9];   /* reciprocal basis, row-major */
  double rot_t[9];   /* transpose of the detector rotation, row-major */
  double p[3];       /* P_Array (m) */
  double px_x, px_y; /* pixel pitch (m) */
  double elo, ehi;   /* energy band (keV) */
  int32_t nr_px_x, nr_px_y;
  int32_t max_nr_spots; /* S */
  int32_t reserved;
} lmb_geometry;

/* One matched orientation of one image. */
typedef struct lmb_survivor {
  uint64_t id;     /* orientation row number */
  int32_t n_spots; /* spots landing on a positive pixel */
  int32_t sum_u8;  /* sum of their uint8 values */
  double tot_int;  /* FP64 intensity sum in record order (the reference's totInt) */
  double score;    /* tot_int * sqrt(n_spots) (LaueMatchingCPU.c:688) */
} lmb_survivor;

typedef struct lmb_engine lmb_engine;

/* Library version and the last error message of the calling thread. */
const char *lmb_version(void);
const char *lmb_last_error(void);

/* Free/total device memory, L2 size and SM count of a device: the budget a
 * server admits image slots against.  No reference counterpart (the
 * reference sizes its DB chunks from cudaMemGetInfo, LaueMatchingGPU.cu:665-687). */
int lmb_device_info(int32_t device, uint64_t *free_bytes, uint64_t *total_bytes,
                    int32_t *l2_bytes, int32_t *sm_count);

/* Detector rotation (Rodrigues of R_Array, LaueMatchingCPU.c:225-239) and the
 * reciprocal basis (calcRecipArray, LaueMatchingHeaders.h:379-436), FP64 in
 * the reference's operation order.  R_Array = (0,0,0) gives NaN, as in the
 * reference. */
int lmb_geometry_init(const double lattice[6], int32_t space_group,
                      const double p_array[3], const double r_array[3],
                      double px_x, double px_y, int32_t nr_px_x,
                      int32_t nr_px_y, double elo, double ehi,
                      int32_t max_nr_spots, lmb_geometry *out);

/* Engine: one device, one geometry, one resident DB, LMB_MAX_SLOTS image
 * slots.  Replaces the device set-up of LaueMatchingGPU.cu:416,665-712 and
 * LaueMatchingGPUStream.cu:998-1075.  survivor_capacity is the per-image
 * survivor buffer (0 = default 262144; the reference caps at 100000 and
 * truncates silently, LaueMatchingGPU.cu:43,754-760). */
int lmb_engine_create(int32_t device, const lmb_geometry *geo,
                      uint64_t survivor_capacity, lmb_engine **out);
int lmb_engine_destroy(lmb_engine *e);
/* cudaStream_t of the engine's compare pass (for external event timing). */
void *lmb_engine_stream(lmb_engine *e);

/* Launch shape of the compare pass: fields = {variant (0 block-barrier ring,
 * 1 warp-specialised, 2 warp-specialised over the compact layout, 3 automatic
 * -- the default: variant 2 while the records that can pass hold at most ~3
 * spots per DB record on average, variant 4 beyond, variant 1 when the
 * compact layout cannot be built --, 4 the compact layout filtered by the
 * cell mask of the pass's frames), tile_sub (32-orientation sub-tiles per
 * tile), stages, consumer warps, blocks per SM, grid multiplier,
 * full_gather, test_consumer_wait_us, cell_consumers, cell_stages,
 * cell_queue}; 0 = default.  cell_consumers, cell_stages and cell_queue (1:
 * the records that can still pass are queued and counted 32 at a time; 0:
 * counted chunk by chunk) shape variant 4 when the automatic variant picks it
 * (the autotuner's dense-DB entry); a pinned variant 4 takes cell_queue from
 * this field too.  full_gather = 1
 * gathers every spot even of records with fewer spots than MinNrSpots (which
 * cannot pass; by default they are skipped; results are identical either
 * way), for measuring the full gather cost.  test_consumer_wait_us (tests
 * only, compact-layout variants) makes the pass's consumer warps wait that
 * long on a barrier nothing arrives at, so the pass gives up and its results
 * report LMB_ERR_TIMEOUT; the engine's device error word is sticky, so that
 * engine reports the timeout from then on.  Written by the autotuner; get
 * returns the shape actually used for this DB.  No reference counterpart
 * (the reference launches <<<ceil(n/1024),1024>>>, LaueMatchingGPU.cu:739-743). */
int lmb_engine_set_tuning(lmb_engine *e, const int32_t *fields, int32_t n_fields);
/* get: fields 0-6 as set, 7: the variant the latest pass ran, 8: the test
 * wait, 9-11: the cell-mask pass's shape for the automatic variant. */
int lmb_engine_get_tuning(lmb_engine *e, int32_t *fields, int32_t n_fields);

/* The compact device layout variant 2 streams: derived from the resident
 * records on the first variant-2 pass (1 byte per record + 4 bytes per
 * on-detector spot, in record order; the reference records stay resident).
 * compact = 1 built, 0 not yet, -1 this DB keeps the reference layout
 * (MaxNrLaueSpots > 255 or tiles too large).  No reference counterpart. */
int lmb_engine_layout_info(lmb_engine *e, int32_t *compact, uint64_t *compact_bytes,
                           int32_t *tiles, int32_t *tile_bytes);

/* lmb_image_load sends a frame whose positive pixels are few (their
 * (uint32 index, value) pairs smaller than half the dense frame) as those
 * pairs, found by a multi-threaded host scan, instead of the whole frame
 * (default on; results are identical either way).  No reference counterpart
 * (the reference copies the dense float frame, LaueMatchingGPUStream.cu:1204). */
int lmb_engine_set_sparse_uploads(lmb_engine *e, int32_t enable);

/* Share (0..1) of the page-locked frames of an lmb_image_load_batch call that
 * are sent dense over the copy engine, enqueued first so that they cross the
 * link while the host scans the others (results are identical either way).
 * Default 0.33: the host scan (~120 GB/s over 16 threads) and the copy engine
 * (~50 GB/s) then finish a batch of 4 MiB frames at about the same time.
 * No reference counterpart. */
int lmb_engine_set_dense_share(lmb_engine *e, double share);

/* Upload a forward cache (n records of 1+2S uint16) into device memory.
 * Replaces the chunked synchronous H2D of LaueMatchingGPU.cu:619-749 and
 * the resident upload of LaueMatchingGPUStream.cu:998-1038. */
int lmb_db_upload(lmb_engine *e, const uint16_t *records, uint64_t n);

/* Forward-simulate the DB on the device from n orientation matrices
 * (row-major 3x3 FP64 each) and nh HKLs (int32 triplets, file order).
 * Replaces the OpenMP forward simulation of LaueMatchingCPU.c:595-667
 * (duplicated at LaueMatchingGPU.cu:478-614, LaueMatchingGPUStream.cu:854-946).
 * Records are identical to the reference's. */
int lmb_db_build(lmb_engine *e, const double *orients, uint64_t n,
                 const int32_t *hkls, int32_t nh);

/* lmb_db_build with flags.  LMB_BUILD_EXACT_FP64 skips the FP32 screen and
 * evaluates every (orientation, HKL) pair in FP64 (a self-check of the
 * screen; same records, slower). */
#define LMB_BUILD_EXACT_FP64 1
int lmb_db_build_ex(lmb_engine *e, const double *orients, uint64_t n,
                    const int32_t *hkls, int32_t nh, uint32_t flags);

/* Same, with orientations generated on the device: uniform random rotations
 * (Shoemake's method) from the counter-based generator keyed by seed, IDs
 * first..first+n-1.  If orients_out is not NULL the matrices are copied to it
 * (n*9 doubles).  For synthetic workloads. */
int lmb_db_build_synthetic(lmb_engine *e, uint64_t seed, uint64_t n,
                           const int32_t *hkls, int32_t nh, double *orients_out);

/* The orientation matrices IDs first..first+n-1 of the synthetic generator
 * above (n*9 doubles to out), bitwise the ones lmb_db_build_synthetic used. */
int lmb_synth_orientations(lmb_engine *e, uint64_t seed, uint64_t first,
                           uint64_t n, double *out);

/* Synthetic builds with flags: LMB_BUILD_EXACT_FP64 as for lmb_db_build_ex;
 * LMB_BUILD_SYNTH_HEX_FZ reduces every generated rotation to the hexagonal
 * (622) fundamental zone -- of its 12 equivalents under the operators of
 * LaueMatchingHeaders.h:111-122 the one with the largest |scalar part|, the
 * reference's own merge criterion -- since the reference never generates
 * zone-restricted DBs (scripts/GenerateOrientations.py:5-9).
 * lmb_synth_orientations_ex gives the same matrices for the same flags. */
#define LMB_BUILD_SYNTH_HEX_FZ 2
int lmb_db_build_synthetic_ex(lmb_engine *e, uint64_t seed, uint64_t n,
                              const int32_t *hkls, int32_t nh, double *orients_out,
                              uint32_t flags);
int lmb_synth_orientations_ex(lmb_engine *e, uint64_t seed, uint64_t first,
                              uint64_t n, double *out, uint32_t flags);

/* Copy records [first, first+count) of the resident DB to the host (to write
 * the ForwardFile, LaueMatchingCPU.c:694-711). */
int lmb_db_download(lmb_engine *e, uint64_t first, uint64_t count,
                    uint16_t *out);
int lmb_db_info(lmb_engine *e, uint64_t *n_orient, int32_t *max_nr_spots);

/* Load one image (NrPxX*NrPxY pixels of dtype LMB_F64 or LMB_F32) into a
 * slot: host->device copy, uint8 quantisation exactly as
 * LaueMatchingCPU.c:356-375 (imScale returned), occupancy-bit update.
 * keep_f64 keeps the float64 copy for LMB_VALUE_F64 passes. */
int lmb_image_load(lmb_engine *e, int32_t slot, const void *pixels,
                   int32_t dtype, int32_t keep_f64, double *im_scale);

/* Load n frames (n <= 64, distinct slots, one dtype) in one call; each slot
 * ends exactly as after lmb_image_load(e, slots[i], frames[i], dtype, 0, ...)
 * and im_scales[i] (optional) receives its imScale.  With sparse uploads on,
 * every frame is read once by a parallel host scan and the pairs of all
 * sparse frames cross the link in one copy, followed by two kernels for the
 * whole batch.  Replaces the per-image H2D of the reference's stream loop
 * (LaueMatchingGPUStream.cu:1201-1205) for a batch of admitted images. */
int lmb_image_load_batch(lmb_engine *e, const int32_t *slots, const void *const *frames,
                         int32_t n, int32_t dtype, double *im_scales);

/* One DB pass over every slot in slot_mask: the compare of
 * LaueMatchingCPU.c:668-690 (replacing the compare kernels
 * LaueMatchingGPU.cu:45-81 and LaueMatchingGPUStream.cu:69-100), survivor
 * compaction and ordering by ID (LaueMatchingCPU.c:781-788).  Asynchronous:
 * results are read with lmb_results.  Passes queue on the engine stream: a
 * pass over other slots may be started before the previous pass's results
 * have been read (they stay valid until a later pass includes the slot). */
int lmb_match(lmb_engine *e, uint64_t slot_mask, int32_t min_nr_spots,
              double min_intensity, int32_t value_mode);

/* Wait for the last pass that included the slot and copy its survivors
 * (ascending id).
 * n_survivors receives the full count; n_pass the reference's nrResults
 * (LaueMatchingCPU.c:686).  Returns LMB_ERR_OVERFLOW when the count exceeded
 * the engine's survivor capacity (the first capacity survivors by ID are
 * then not guaranteed: recreate the engine with a larger capacity). */
int lmb_results(lmb_engine *e, int32_t slot, lmb_survivor *out,
                uint64_t out_capacity, uint64_t *n_survivors, uint64_t *n_pass);

/* lmb_results for several slots at once: survivors of slots[0..nslots) are
 * written back to back into out (slot order as given, each ascending id);
 * counts[i] / n_pass[i] receive each slot's survivor and pass counts.
 * Returns LMB_ERR_OVERFLOW (counts filled, nothing copied) when out_capacity
 * is too small or a slot overflowed the engine capacity. */
int lmb_results_batch(lmb_engine *e, const int32_t *slots, int32_t nslots, lmb_survivor *out,
                      uint64_t out_capacity, uint64_t *counts, uint64_t *n_pass);

/* Device time of the last pass in milliseconds (CUDA events on the engine
 * stream): compare kernel, ordering kernel. */
int lmb_last_pass_ms(lmb_engine *e, float *compare_ms, float *order_ms);

/* Bytes the engine has moved host->device and device->host since it was
 * created (DB and orientation uploads, frames as sent -- sparse or dense --,
 * status words, survivors, downloads).  The reference prints its transfer
 * sizes and times per chunk (LaueMatchingGPU.cu:683-717,747); these counters
 * are the engine's equivalent for a caller's end-to-end accounting. */
int lmb_engine_bytes(lmb_engine *e, uint64_t *h2d_bytes, uint64_t *d2h_bytes);

/* ---- host post-stage ------------------------------------------------------
 * Duplicate merge (mergeDuplicateOrientations, LaueMatchingHeaders.h:969-1065)
 * and refinement + output text (fitAndWriteOrientations, :1072-1153) for the
 * survivors of one image, as LaueMatchingCPU.c:735-809 and
 * LaueMatchingGPUStream.cu:436-533 call them.  The refinement optimiser
 * evaluates the objective once at the coarse orientation (NLopt is not
 * available here; the reference built with an evaluate-once NLopt writes the
 * same text).  Grains are written in grain order. */
typedef struct lmb_post_params {
  double lattice[6];     /* LatticeParameter (nm, degrees) */
  int32_t space_group;   /* SpaceGroup */
  int32_t max_nr_spots;  /* unused: the fit uses 3*geometry max_nr_spots */
  double tol_latc[6];    /* tol_LatC */
  double tol_c_over_a;   /* tol_c_over_a (non-zero zeroes tol_latc) */
  double max_angle;      /* MaxAngle (degrees) */
  int32_t min_nr_spots;  /* MinNrSpots (CLI) or MinGoodSpots (daemon) */
  int32_t image_num;     /* > 0: prepend the ImageNr column (daemon format) */
  int32_t num_threads;   /* host threads */
  int32_t optimizer;     /* 0 = evaluate once (the reference built without NLopt);
                            1 = this library's bounded Nelder-Mead, all grains at once
                            (lmb_refine_fit, 200 evaluations; not NLopt's steps) */
  int32_t max_results;   /* candidates kept for the merge, top by score;
                            0 = the reference's cap MERGE_MAX_RESULTS 50000 */
  int32_t merge_on_device; /* k > 0: for 1024 or more candidates, the duplicate merge's
                              pair matrix and greedy pass run on CUDA device k-1 (same
                              clusters; at most 200000 candidates), and with optimizer 1
                              and 2048 or more grains the refinement's evaluations too
                              (same fits); 0: all on the host */
} lmb_post_params;

typedef struct lmb_post_output {
  char *solutions; /* solutions.txt lines (no header), NUL terminated */
  uint64_t solutions_len;
  char *spots; /* spots.txt lines (no header) */
  uint64_t spots_len;
  int32_t n_unique; /* clusters after the merge ("Unique Orientations") */
} lmb_post_output;

/* ids/scores: the image's survivors in ascending id (the CPU collection
 * order); orients: all n_orients matrices; image: the float image. */
int lmb_post_process(const lmb_geometry *geo, const lmb_post_params *pp,
                     const double *orients, uint64_t n_orients,
                     const uint64_t *ids, const double *scores,
                     int64_t n_results, const float *image,
                     const int32_t *hkls, int32_t nh, lmb_post_output *out);
void lmb_post_free(lmb_post_output *out);

/* The duplicate merge alone (mergeDuplicateOrientations, LaueMatchingHeaders.h:
 * 998-1065, after its cap): candidates rows[0..n) with scores, in input order,
 * clustered greedily by misorientation <= max_angle (degrees) under the space
 * group's symmetry.  Out: n_clusters, and per cluster the kept row, its score
 * and the candidate count (arrays of n entries).  device >= 0 with n >= 1024:
 * the pair matrix and the greedy pass run on that CUDA device (at most 200000
 * candidates); pairs whose device angle lies within max(host_band, a 1e-12
 * relative band) of the float rounding boundary at max_angle are decided with
 * the host function.  device < 0: the host loop.  Same clusters either way. */
int lmb_merge_clusters(int32_t device, int32_t space_group, double max_angle,
                       double host_band, const double *orients, uint64_t n_orients,
                       const uint64_t *rows, const double *scores, int64_t n,
                       int32_t num_threads, int32_t *n_clusters, uint64_t *best_rows,
                       double *best_scores, int32_t *counts);

/* ---- batched orientation refinement ----------------------------------------
 * FitOrientation (LaueMatchingHeaders.h:696-801) for many grains at once, as
 * fitAndWriteOrientations (:1072-1153) sets it up: per grain the Euler angles
 * of its coarse matrix (OrientMat2Euler), the HKLs valid there
 * (prefilterHKLs, :513-561, with the parameters' lattice), the start point
 * and box (Euler +-3 degrees, lattice entries x (1 +- tol_LatC), or c/a x
 * (1 +- tol_c_over_a)), and problem_function (:640-694 with
 * calcOverlapFiltered :564-636) as the objective: -(nrPos * sqrt(sum)) over
 * at most 3 x max_nr_spots spots.  device >= 0: objective evaluations run on
 * that CUDA device, one launch per round for all grains; device < 0: on
 * pp->num_threads host threads.  Both give bit-identical values.  The
 * images are float frames of nr_px_y rows of nr_px_x (image[py * nr_px_x +
 * px]), copied at lmb_refine_set_images; set_images drops the grains. */
typedef struct lmb_refine lmb_refine;
int lmb_refine_create(int32_t device, const lmb_geometry *geo, const lmb_post_params *pp,
                      const int32_t *hkls, int32_t nh, lmb_refine **out);
int lmb_refine_destroy(lmb_refine *r);
/* n: the fit's dimension count (3 + lattice entries with a tolerance, or 4) */
int lmb_refine_dims(lmb_refine *r, int32_t *n);
int lmb_refine_set_images(lmb_refine *r, const float *const *frames, int32_t n_images);
/* orients[n_grains][9]: coarse orientation matrices; image[n_grains]: frame
 * index of each grain; n_valid (optional, [n_grains]): prefiltered HKL counts */
int lmb_refine_set_grains(lmb_refine *r, const double *orients, const int32_t *image,
                          int32_t n_grains, int32_t *n_valid);
/* start points and box of every grain, [n_grains][n] each (any may be NULL) */
int lmb_refine_start(lmb_refine *r, double *x0, double *lower, double *upper);
/* problem_function at m points: x[m][n] of grain[m] -> objective[m] */
int lmb_refine_evaluate(lmb_refine *r, const int32_t *grain, const double *x, int64_t m,
                        double *objective);
/* Fit every grain.  optimizer 0: evaluate once at the start point (the
 * reference built with an evaluate-once NLopt stand-in gives the same
 * result); 1: this library's bounded Nelder-Mead, all grains in lockstep,
 * at most max_eval evaluations per grain, stopping at relative changes of
 * 1e-6 in value or position (NLopt is not available; NLopt's own
 * NELDERMEAD / BOBYQA take other steps).  The start simplex steps each
 * coordinate by init_step x its box width (<= 0: 0.02).  Out: x_fit[n_grains][n],
 * overlap[n_grains] (= -objective at x_fit), evals[n_grains] (optional). */
int lmb_refine_fit(lmb_refine *r, int32_t optimizer, int32_t max_eval, double init_step,
                   double *x_fit, double *overlap, int32_t *evals);
/* Of the last evaluate / fit call: points evaluated, rounds (launches on a
 * device), summed device time of the objective kernel (0 on the host). */
int lmb_refine_last_stats(lmb_refine *r, int64_t *points, int32_t *rounds, float *kernel_ms);
/* What the calling thread's last lmb_post_process refined (optimizer 1):
 * device -2 = no refinement, -1 = host threads, else the device ordinal;
 * points, rounds and objective-kernel time as lmb_refine_last_stats gives
 * them.  The post-stage keeps its refinement handles between calls (no
 * allocation per image once a handle exists for that device, geometry,
 * parameters and HKL list). */
int lmb_post_last_refine_stats(int32_t *device, int64_t *points, int32_t *rounds,
                               float *kernel_ms);

/* ---- survivor ordering that allocates nothing ------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves (code running inside another framework's memory pool, or
 * on a thread that must not take cudaMalloc's implicit device
 * synchronisation) but hold device buffers: sorts d_in[0..n) (unsorted
 * survivors) by orientation id, ties by position, into d_out (the two ranges
 * must not overlap), with the same order as lmb_results delivers, on
 * `stream` (a cudaStream_t; NULL = legacy default stream).  Ids of 2^40 and
 * above are ordered too (by a slower comparison that reads the ids from
 * d_in).  Makes no cudaMalloc/cudaFree call: lists above 8192
 * entries use a fixed 8 MiB device array inside the library as key scratch,
 * which every GPU that loads the library holds until the process exits.
 * n above LMB_NOALLOC_ORDER_MAX is rejected with LMB_ERR_INVALID.  The first
 * call on a device resolves that array's address (cudaGetSymbolAddress) and
 * sets the kernel's shared-memory limit; make it before any stream capture.
 * That set-up is kept for the life of the process: a cudaDeviceReset of the
 * device afterwards is not supported (later calls would launch with the
 * stale address).  All calls share the one scratch array, so calls that
 * overlap on the GPU (other streams, other threads) race: serialise them. */
#define LMB_NOALLOC_ORDER_MAX (1u << 20)
int lmb_order_survivors_noalloc(const lmb_survivor *d_in, uint64_t n,
                                lmb_survivor *d_out, void *stream);

/* ---- frame preprocessing ----------------------------------------------------
 * Replaces laue_index/preprocess.py:221-338 (preprocess_image; called by
 * scripts/laue_image_server.py:66-80 and scripts/RunImage.py:150-299) as the
 * reference runs with numpy, scipy and OpenCV and without diplib or
 * scikit-image: background = scipy's square median filter
 * (preprocess.py:42-65), subtraction clipped at 0, threshold
 * (thresholds.py:29-110; "otsu" falls back to the adaptive noise floor),
 * float64 -> uint16, 8-connected components numbered as OpenCV numbers them
 * (preprocess.py:136-151), components below min_area removed and the
 * intensity-weighted centre of each kept one (preprocess.py:154-188), then
 * the Gaussian blur of the filtered frame (preprocess.py:315-329).  Every
 * output is identical to the reference's; the blur weights come from the
 * caller (numpy's exp, as scipy builds them).  One handle per (device,
 * frame size); calls on a handle are not re-entrant. */
typedef struct lmb_pre lmb_pre;

#define LMB_U16 3 /* uint16 detector frame (preprocessing input only) */

#define LMB_THR_ADAPTIVE 0   /* median(nz) + 4 * 1.4826 * MAD(nz), at least 1 */
#define LMB_THR_PERCENTILE 1 /* np.percentile(frame, threshold_percentile), linear */
#define LMB_THR_FIXED 2      /* threshold_value */

typedef struct lmb_pre_params {
  int32_t threshold_method;    /* LMB_THR_* (cfg threshold_method) */
  int32_t min_area;            /* cfg min_area */
  double threshold_value;      /* cfg threshold_value (fixed method) */
  double threshold_percentile; /* cfg threshold_percentile */
  double override_thresh;      /* > 0: fixed threshold of this value (preprocess.py:280-283) */
} lmb_pre_params;

typedef struct lmb_pre_counts {
  double threshold;  /* threshold applied (pixels <= it are zeroed) */
  double min_dist2;  /* smallest squared distance between two kept centres; +inf below 2 */
  int32_t n_labels;  /* OpenCV's nlabels: components + 1 */
  int32_t n_centres; /* components with area >= min_area */
} lmb_pre_counts;

int lmb_pre_create(int32_t device, int32_t nr_px_y, int32_t nr_px_x, lmb_pre **out);
int lmb_pre_destroy(lmb_pre *p);

/* scipy.ndimage.median_filter(frame, size) applied `passes` times (mode
 * reflect), exact for any float64 values (preprocess.py:63-65).  The result
 * becomes the handle's background and is copied to `out` (may be NULL).
 * Sizes reaching 8x a frame side (>1 pixel) are refused: scipy's border
 * handling stops being a mirror there. */
int lmb_pre_median(lmb_pre *p, const void *frame, int32_t dtype, int32_t size, int32_t passes,
                   double *out);
/* The background subtracted from the following frames (float64 [y][x]);
 * NULL = zeros.  Kept on the device until replaced. */
int lmb_pre_set_background(lmb_pre *p, const double *background);
int lmb_pre_get_background(lmb_pre *p, double *out);

/* Steps up to the centres for one raw frame (dtype LMB_F64/F32/U16/U8):
 * max(frame - background, 0), threshold, uint16 cast, components, small
 * ones removed, centres.  Results stay on the device for the calls below. */
int lmb_pre_segment(lmb_pre *p, const void *frame, int32_t dtype, const lmb_pre_params *prm,
                    lmb_pre_counts *counts);
/* The same from an already thresholded uint16 frame (find_connected_components
 * + filter_small_components, preprocess.py:136-188). */
int lmb_pre_segment_thresholded(lmb_pre *p, const uint16_t *thresholded, int32_t min_area,
                                lmb_pre_counts *counts);
/* Centres of the last segment in label order: [label, cx, cy, area] per row
 * (up to cap rows); bboxes/areas of all components [x, y, w, h, area] (up to
 * cap rows; may be NULL). */
int lmb_pre_centres(lmb_pre *p, double *centres, int32_t cap);
int lmb_pre_stats(lmb_pre *p, int32_t *stats, int32_t cap);
/* Frames of the last segment; any pointer may be NULL. */
int lmb_pre_images(lmb_pre *p, uint16_t *thresholded, int32_t *labels, uint16_t *filt_img,
                   int32_t *filt_labels);
/* Gaussian blur of the last segment's filtered frame with weights[0..2r]
 * (scipy.ndimage.gaussian_filter: axis 0 then axis 1, mirrored borders) into
 * host memory as float64 (LMB_F64) or float32 (LMB_F32, the image server's
 * wire format, laue_image_server.py:79). */
int lmb_pre_blur(lmb_pre *p, const double *weights, int32_t radius, void *out, int32_t out_dtype);

/* The blur of lmb_pre_blur straight into image slot `slot` of an engine on the
 * same device, quantised there as lmb_image_load quantises a host frame, with no
 * host round trip of the blurred frame.  frame_dtype is the form in which the
 * reference hands the blurred frame to its matcher: LMB_F32 for the stream
 * daemon (the image server sends float32, laue_image_server.py:79), LMB_F64 for
 * the LaueMatchingGPU executable (RunImage writes float64, RunImage.py:290-292);
 * the slot then holds exactly what loading that frame from the host would give.
 * im_scale (may be NULL) receives the slot's imScale.  No reference
 * counterpart: the reference moves the blurred frame through a file or TCP. */
int lmb_pre_blur_to_slot(lmb_pre *p, const double *weights, int32_t radius, lmb_engine *e,
                         int32_t slot, int32_t frame_dtype, double *im_scale);

/* Device times (ms, CUDA events on the handle's stream) of the stages of the
 * last calls: [0] frame upload, [1] subtraction + threshold, [2] components,
 * centres and closest pair, [3] blur, [4] blur download, [5] median frame
 * upload, [6] median ranks (last pass), [7] median kernel (last pass).  No
 * reference counterpart. */
#define LMB_PRE_STAGES 8
int lmb_pre_timings(lmb_pre *p, float *ms, int32_t n);

/* Page-locked host buffers, so image uploads run at full link speed.  No
 * reference counterpart (the reference pins per-stream buffers internally,
 * LaueMatchingGPUStream.cu:1041-1075). */
int lmb_host_alloc(uint64_t bytes, void **out);
int lmb_host_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* LMB200_H */
