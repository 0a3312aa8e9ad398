/*
 * extremz.h -- C ABI of the B200 ExtreM correction library (libextremz.so).
 *
 * The library corrects a lossy-decompressed scalar field so that its critical
 * points and its ascending / descending manifold labels match the original,
 * by lowering values within the absolute error bound.  It is the drop-in for
 * the reference's correction call:
 *   - the GPU correction driver, main() of src/ExtreM_cuda.cu:4954-6078
 *     (classification, manifolds, c_loops / r_loops / s_loops / saddle_loops
 *     and the outer loop), and
 *   - the CPU correction sequence of main.cpp:65-446 over the host API
 *     include/api/ExtreM.h:43-123 (getdata, classifyAllVertices,
 *     ComputeDescendingManifold / ComputeAscendingManifold, c_loops, r_loops,
 *     s_loops, saddle_loops).
 * Buffers are caller-owned plain pointers; no C++ or torch types cross this
 * boundary.  Every entry point returns a status code instead of exiting.
 */
#ifndef EXTREMZ_H
#define EXTREMZ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: extremz_report times twelve kernel classes (the first manifold round's
 * directions and jumps apart from the later rounds'). */
#define EXTREMZ_ABI_VERSION 2

typedef enum {
  EXTREMZ_OK = 0,
  EXTREMZ_ROUND_CAP = 1,      /* a round cap was hit before zero mismatch */
  EXTREMZ_BAD_ARG = 2,
  EXTREMZ_OOM = 3,
  EXTREMZ_CUDA_ERR = 4,
  EXTREMZ_DEVICE_TIMEOUT = 5, /* a device-side iteration limit was hit */
  EXTREMZ_NO_DEVICE = 6,
  EXTREMZ_TOO_LARGE = 7,      /* beyond EXTREMZ_NOALLOC_MAX_VOXELS (noalloc entry point),
                                 or beyond a server's whole HBM budget */
  EXTREMZ_PENDING = 8         /* server request still queued or running */
} extremz_status;

typedef enum { EXTREMZ_F32 = 0, EXTREMZ_F64 = 1 } extremz_dtype;

/*
 * Correction parameters.  The reference takes them on the command line of
 * src/ExtreM_cuda.cu (:4958-4963, :5015-5018) and hard-codes the rest:
 *   bound      absolute error bound; the reference computes
 *              (max - min) * er of the original field (:229-232)
 *   thr        persistence filter of the ascending rows, sim * (max - min) (:231)
 *   q          step divisor and edit-counter threshold (:4962, :5015)
 *   edit_type  0: fixed step -bound/q gated by the edit counter;
 *              1: midpoint step toward input - bound (:4963, :3061-3111)
 *   max_outer, max_cloop_rounds
 *              caps the reference does not have (its loops at :3961 and
 *              :5603 are unbounded); hitting one returns EXTREMZ_ROUND_CAP
 *   final_join run the unconditional saddle_loops_join after the loop (:5997)
 *   preserve_join
 *              preserve_join_tree of the reference (:4969, false there)
 */
typedef struct {
  double bound;
  double thr;
  int q;
  int edit_type;
  int max_outer;
  int max_cloop_rounds;
  int final_join;
  int preserve_join;
  int flags;          /* EXTREMZ_FLAG_* */
  int device_iter_cap; /* device-side iteration limit of pointer jumping and path
                          walks; 0 = the field's voxel count (never reached by a
                          valid path).  Reaching it sets report.error_bits and
                          returns EXTREMZ_DEVICE_TIMEOUT. */
  /* Launch-shape knobs, picked per dtype and size class by the project's
   * autotuner (extrem_z_b200/autotune.py); results do not depend on them.
   * 0 = defaults (8 and 4). */
  int tune_blocks_per_sm; /* blocks per SM of the grid-stride kernels, 1..32 */
  int tune_pass_chunk;    /* 1024-id blocks per saddle-pass work item, 1..64 */
  int reserved[2];
} extremz_params;

/* flags: time kernel launches with CUDA events, per kernel class, into
 * extremz_report.prof_ms / prof_launches.  Bits from
 * EXTREMZ_PROFILE_CLASS_SHIFT up select the classes to time (none set = all),
 * so that a benchmark can time only its dominant kernel. */
#define EXTREMZ_FLAG_PROFILE 1
#define EXTREMZ_PROFILE_CLASS_SHIFT 8
/* flags: load halo tiles with plain loads instead of TMA bulk tensor copies
 * (TMA is used whenever the field's base is 16-byte aligned and its row stride
 * W * sizeof(value) is a multiple of 16 bytes). */
#define EXTREMZ_FLAG_NO_TMA 2
/* flags: resolve the wrong-neighbour flags (get_wrong_split_neighbors /
 * get_wrong_join_neighbors, src/ExtreM_cuda.cu:2400-2513) sequentially in
 * ascending saddle id instead of the default lockstep order.  The reference
 * flags with a check-then-set from concurrent threads, so its runs can differ.
 * By default a neighbour two saddles share goes to the saddle that meets it at
 * the earlier neighbour index, which is what the reference's launch does when
 * its threads advance through their neighbour loops in step: its output on
 * the 256^3 and 512^3 benchmark fields and on every pinned test field whose
 * runs agree.  The ascending order gives the same result wherever no two
 * saddles contend for a neighbour. */
#define EXTREMZ_FLAG_WN_ASCENDING 4

/* Kernel classes of extremz_report.prof_*: 0 setup (classification, labels and
 * rows of the original field), 1 fused classification + mismatch detection,
 * 2 steepest directions and 3 pointer jumping of the decompressed field in the
 * manifold rounds after a correction's first (changed tiles, touched chains),
 * 4 proposals, 5 apply, 6 saddle pass (decompressed rows and wrong-neighbour
 * seeds), 7 wrong-neighbour resolution, 8 path walks, 9 everything else,
 * 10 steepest directions and 11 pointer jumping of the decompressed field in
 * a correction's first manifold round (every tile, every vertex). */
#define EXTREMZ_NUM_KCLASS 12

/* Outcome of one correction. counters[] are the eleven host counters of the
 * reference's loop test (:5603-5605) at exit: wrong split / join neighbours,
 * false max / min / saddle counts, wrong_max(2), wrong saddle, wrong_min(2),
 * wrong join saddle. */
typedef struct {
  int status;
  int outer_iters;
  int cloop_rounds;
  int manifold_rounds;
  int counters[11];
  int error_bits;
  long long kernel_launches;          /* kernels this call launched */
  float prof_ms[EXTREMZ_NUM_KCLASS];  /* with EXTREMZ_FLAG_PROFILE */
  int prof_launches[EXTREMZ_NUM_KCLASS];
  int manifold_reused;  /* manifold rounds whose inputs were unchanged since the
                           previous round, so its results were kept */
  int cp_counts[4];     /* original 2-saddles, 1-saddles, maxima, minima */
  int graph_launches;   /* ticks launched as one CUDA graph (see extremz_correct_device) */
  long long host_bytes_back;  /* extremz_correct_host: bytes copied device -> host */
} extremz_report;

typedef struct extremz_ctx_s extremz_ctx;

/* ABI version of the loaded library (EXTREMZ_ABI_VERSION). */
int extremz_version(void);

/* Reference defaults: q = 4, edit_type = 1, thr = 0, final join on. */
void extremz_default_params(extremz_params* p);

/* A context owns the device workspace (grown on demand, reused across calls)
 * for one device.  Calls on one context must not overlap. */
extremz_status extremz_ctx_create(int device, extremz_ctx** out);
void extremz_ctx_destroy(extremz_ctx* ctx);

/*
 * Correct d_decp in place.  d_orig and d_decp are device pointers to
 * width*height*depth values of dtype (x fastest).  stream is a cudaStream_t
 * (NULL = legacy default stream).  trace (host, optional) receives records of
 * four int32 (phase, counter, counter, counter) for debugging; trace_cap is its
 * length in int32.  The launches of one step of the control flow ("tick") that
 * repeat an earlier step's exactly run as one CUDA graph, captured the third
 * time they occur and kept in the context (not when the caller's stream is
 * itself being captured).  With EXTREMZ_FLAG_PROFILE the timed launches' events
 * are part of the graphs, so profiling does not change how ticks launch.
 * Replaces: main() of src/ExtreM_cuda.cu:5508-5997 (the correction proper, with
 * input and decompressed field already resident on the device).
 */
extremz_status extremz_correct_device(extremz_ctx* ctx, const void* d_orig, void* d_decp,
                                      int dtype, int width, int height, int depth,
                                      const extremz_params* params, extremz_report* report,
                                      void* stream, int32_t* trace, int trace_cap);

/*
 * Mismatch census of a (corrected) field d_field against the original d_orig,
 * both on the device: the eleven loop-test counters, in the order of
 * extremz_report.counters, evaluated once with no edit (d_field is only read).
 * The counters are: wrong split / join neighbours (manifold-label mismatches),
 * false maxima / minima / saddles (critical-point mismatches), wrong maxima,
 * wrong maxima (second), wrong saddles, wrong minima, wrong minima (second),
 * wrong join saddles.  The reference's loop evaluates the wrong-extremum and
 * wrong-saddle counters only when the wrong-neighbour counts are zero, and the
 * join ones only with preserve_join_tree; the census evaluates all of them.
 * Synchronises the stream.
 * Replaces: the loop test's counters (src/ExtreM_cuda.cu:5589-5605) read on
 * the final field, which the reference never does after its unconditional
 * saddle_loops_join (:5997).
 */
extremz_status extremz_mismatch_census(extremz_ctx* ctx, const void* d_orig, const void* d_field,
                                      int dtype, int width, int height, int depth, double thr,
                                      int32_t* counters, void* stream);

/*
 * Same with host buffers: copies both fields to the device, corrects, and
 * writes the corrected field back into h_decp.  h_decp still holds the
 * decompressed field at that point, so only the voxels whose value changed
 * travel back (their ids and values, stored into h_decp on the host) unless
 * more than 1/16 of the voxels changed, when the whole field is copied;
 * report->host_bytes_back gives the bytes copied.
 * Replaces: the correction sequence of main.cpp:65-446 (host arrays in,
 * corrected decp_data out, saved by saveArrayToBin at main.cpp:507).
 */
extremz_status extremz_correct_host(extremz_ctx* ctx, const void* h_orig, void* h_decp,
                                    int dtype, int width, int height, int depth,
                                    const extremz_params* params, extremz_report* report,
                                    void* stream);

/*
 * Edit stream of a correction: what the reference's cost() (edit_type 0,
 * src/ExtreM_cuda.cu:4557-4675) and floating_point_cost() (edit_type 1,
 * :4677-4797) compute from the decompressed and corrected fields, before
 * their zstd step.  A voxel is edited when its corrected value differs from
 * its decompressed value.
 *   edit_type 0: index = every voxel's edit counter (0 when not edited),
 *                3 bits per voxel, LSB first (encodeTo3BitBitmap :4282-4312);
 *                edits = -(decp - (orig - bound)) of the voxels whose counter
 *                reached q, in id order.
 *   edit_type 1: index = the edited voxels' ids, delta-coded, int32
 *                (get_diff_index :4315-4323); edits = -(decp - (orig - bound))
 *                of every edited voxel, in id order.
 * index / edits are device buffers of the caller (edits in the field's dtype);
 * extremz_edit_stream_caps gives sizes that always suffice.
 */
typedef struct {
  void* index;
  long long index_cap;   /* bytes */
  void* edits;
  long long edits_cap;   /* bytes */
  /* filled in: */
  long long index_bytes, edit_bytes;
  long long edited;      /* voxels whose value changed */
  long long n_edits;     /* entries of the edit stream */
  double psnr_before;    /* decompressed field against the original (calculatePSNR :4273) */
  double psnr_after;     /* corrected field against the original */
  int reserved[4];
} extremz_edit_stream;

/* Buffer sizes that hold any edit stream of a field of this shape. */
extremz_status extremz_edit_stream_caps(int dtype, int width, int height, int depth, int edit_type,
                                        long long* index_cap, long long* edits_cap);

/*
 * extremz_correct_device, then the edit stream of the correction into es.
 * Returns EXTREMZ_BAD_ARG when a stream buffer is too small (es holds the
 * sizes needed) or, for edit_type 0, when q > 7 (counters need more than
 * three bits; the reference then writes an empty stream).
 * Replaces: the correction and the cost() / floating_point_cost() call of
 * main() (src/ExtreM_cuda.cu:5508-6063).
 */
extremz_status extremz_correct_encode(extremz_ctx* ctx, const void* d_orig, void* d_decp, int dtype,
                                      int width, int height, int depth,
                                      const extremz_params* params, extremz_report* report,
                                      void* stream, extremz_edit_stream* es);

/*
 * Per-vertex critical-point type (int8: 0 minimum, 1 1-saddle, 2 2-saddle,
 * 3 both, 4 maximum, 5 regular, -1 no table entry) and the roots of the
 * steepest-ascent (d_ds, the maximum a vertex ascends to) and steepest-descent
 * (d_as, the minimum) paths of every vertex, into caller device buffers of
 * width*height*depth entries (any of the three may be NULL).  Ties are broken
 * by vertex id.  Synchronises the stream.
 * Replaces: classifyVertex_CUDA (src/ExtreM_cuda.cu:3720-3911) and
 * ComputeDirection + ComputeDescendingManifold / ComputeAscendingManifold
 * (:1464-1611), which the host API exposes as classifyAllVertices and
 * ComputeDescendingManifold / ComputeAscendingManifold
 * (include/api/ExtreM.h:52-54).
 */
extremz_status extremz_classify(extremz_ctx* ctx, const void* d_field, int dtype, int width,
                                int height, int depth, int8_t* d_type, int32_t* d_ds,
                                int32_t* d_as, void* stream);

/*
 * Merge-tree persistence pairs of a field (device pointer), for checking that
 * a correction kept the topology: the split tree pairs every maximum with the
 * vertex where its superlevel component merges into an older one, the join
 * tree every minimum with the vertex where its sublevel component merges; the
 * global maximum pairs with the global minimum and vice versa.  Merge vertices
 * are found from their links (upper / lower link with two or more
 * components), so thin grids (2-D slices) are covered too.  Pairs are (partner vertex, extremum vertex),
 * two int32 each, one per maximum (d_max_pairs) and per minimum
 * (d_min_pairs), extrema ordered by value then id (ascending for maxima,
 * descending for minima).  Caps are in int32 entries; n_max / n_min receive
 * the numbers of extrema (BAD_ARG when a buffer is too small).
 * Replaces: constructPersistencePairs (src/ExtreM.cpp :2132-2249), called by
 * compute_MergeT (:2930-2952) -- the same extremum-graph pairing, on the
 * field's own critical points and manifold labels.
 */
extremz_status extremz_persistence_pairs(extremz_ctx* ctx, const void* d_field, int dtype,
                                        int width, int height, int depth, int32_t* d_max_pairs,
                                        long long max_pairs_cap, int32_t* d_min_pairs,
                                        long long min_pairs_cap, long long* n_max,
                                        long long* n_min, void* stream);

/*
 * The same pairs, plus per extremum the vertex of the extremum it merges into
 * at its partner vertex (d_max_parent / d_min_parent, one int32 per extremum
 * in the same order, each buffer at least half the pair buffer's cap; either
 * may be NULL): the largest maximum (smallest minimum) of its saddle's row
 * when it pairs, the second element of the reference's maximaTriplets
 * (constructPersistencePairs :2183-2187).  The global extremum holds itself.
 * The branch decomposition of constructMergeTree (:1863-1918) follows from
 * these by compressing each parent to the first one still alive at the
 * extremum's partner (extrem_z_b200.api.merge_tree_branches).
 */
extremz_status extremz_persistence_tree(extremz_ctx* ctx, const void* d_field, int dtype, int width,
                                       int height, int depth, int32_t* d_max_pairs,
                                       long long max_pairs_cap, int32_t* d_min_pairs,
                                       long long min_pairs_cap, int32_t* d_max_parent,
                                       int32_t* d_min_parent, long long* n_max, long long* n_min,
                                       void* stream);

/* zstd-compressed size of a host buffer at the given level (the reference
 * compresses both streams with the zstd tool at its default level 3), from
 * the system's libzstd.so.1 loaded at run time; -1 when it is not present. */
long long extremz_zstd_size(const void* host, long long bytes, int level);

/* One field of a batch: device pointers, its own dtype, shape and parameters. */
typedef struct {
  const void* orig;
  void* decp;
  int dtype;
  int width, height, depth;
  extremz_params params;
} extremz_field;

/*
 * Correct n fields in place, each as extremz_correct_device would, with one
 * launch per kernel serving every field that is at the same phase.  Fields
 * of different dtype, shape and parameters mix freely; each field's result
 * is bit-identical to correcting it alone.  Up to 64 fields of each dtype are
 * in flight; the rest are admitted as earlier ones finish, and while device
 * memory is short.  reports (optional) has n entries; reports[0].kernel_launches
 * counts the whole batch's launches.
 * Replaces: a loop over fields of main() of src/ExtreM_cuda.cu:5508-5997 (the
 * reference corrects one field per process run).
 */
extremz_status extremz_correct_batch(extremz_ctx* ctx, const extremz_field* fields, int n,
                                     extremz_report* reports, void* stream);

/*
 * Serving: request loops on their own threads and CUDA streams.  Requests
 * (device fields) arrive at any time; a loop admits them, in arrival order,
 * while the device footprint of the admitted jobs (workspace plus both
 * fields) stays within the HBM budget and a slot is free, and runs every
 * admitted job together: one launch per kernel serves all jobs at the same
 * phase (continuous batching).  Two loops ("lanes") split requests by size;
 * the small-request lane's streams have the higher priority.  A job's field, labels and edit state stay on
 * the device from admission to completion.  Each result is bit-identical to
 * correcting the field alone.
 * No counterpart in the reference (one field per process run, main() of
 * src/ExtreM_cuda.cu:4954-6078).
 */
typedef struct {
  long long hbm_budget_bytes; /* admission budget; 0 = 120 GB */
  long long reserve_bytes;    /* device memory mapped for workspaces at creation
                                 (0 = on demand); at most the budget */
  long long split_voxels;     /* requests above this many voxels go to the
                                 lower-priority lane; 0 = 4 Mi, < 0 = one lane */
  int max_jobs;               /* jobs in flight per dtype and lane, 1..64; 0 = 64 */
  int reserved[7];
} extremz_server_config;

typedef struct {
  long long submitted, completed, queued, running;
  long long bytes_in_use, peak_bytes_in_use;
  long long ticks, kernel_launches;
  int peak_running;
  int reserved[7];
} extremz_server_stats;

typedef struct extremz_server_s extremz_server;

extremz_status extremz_server_create(int device, const extremz_server_config* cfg,
                                     extremz_server** out);
/* Finishes the jobs already admitted, fails the queued ones, then stops. */
void extremz_server_destroy(extremz_server* srv);

/*
 * Queue one field.  Its buffers must stay valid until the request completes.
 * stream: the caller's stream on which the field's contents were produced;
 * the server's work on the field starts after the work queued on it so far.
 * Returns EXTREMZ_TOO_LARGE for a field whose footprint exceeds the budget.
 */
extremz_status extremz_server_submit(extremz_server* srv, const extremz_field* field,
                                     void* stream, long long* ticket);

/* EXTREMZ_PENDING while queued or running; else the request's final status,
 * its report and its latency (submission to completion, host clock), after
 * which the ticket is forgotten. */
extremz_status extremz_server_poll(extremz_server* srv, long long ticket, extremz_report* report,
                                   double* latency_ms);

/* As poll, waiting up to timeout_ms (< 0: without limit) for completion. */
extremz_status extremz_server_wait(extremz_server* srv, long long ticket, int timeout_ms,
                                   extremz_report* report, double* latency_ms);

void extremz_server_get_stats(extremz_server* srv, extremz_server_stats* out);

/* Device bytes a server charges a request of this shape and dtype against its
 * budget: the worst-case workspace of the correction plus both fields. */
long long extremz_job_footprint(int dtype, int width, int height, int depth);

/*
 * Allocation-free variant of extremz_correct_device, for callers that cannot
 * allocate device memory when they correct a field: applications whose
 * allocator owns all of the device memory, so that a cudaMalloc of the
 * library's own would fail or break its accounting, and real-time code that
 * forbids allocation after start-up because an allocation can block.
 * No counterpart in the reference: it always allocates its ~60 device arrays
 * in main() (src/ExtreM_cuda.cu:4997-5185).
 *
 * The whole workspace is a static device array sized for at most
 * EXTREMZ_NOALLOC_MAX_VOXELS voxels (about 31 MB, held by every GPU that loads
 * the library until the process exits); larger fields return
 * EXTREMZ_TOO_LARGE without touching the device.  The call makes no
 * cudaMalloc, cudaFree or other allocating call.  Inputs and outputs are the
 * caller's, as for extremz_correct_device, on the current device and the given
 * stream.  The first call on a device looks up the static arrays' device
 * addresses and uploads the lookup table (synchronously); make that first call
 * before any stream capture.  Every call synchronises the stream: it reads the
 * loop counters back between rounds and waits for its kernels before it
 * returns, errors included.  All calls on a device share the one
 * workspace, so calls that overlap on the GPU race: issue them one after
 * another.  Every call clears what it needs zeroed itself.  Profiling and
 * tracing are off.
 */
#define EXTREMZ_NOALLOC_MAX_VOXELS 65536
extremz_status extremz_correct_device_noalloc(const void* d_orig, void* d_decp, int dtype,
                                              int width, int height, int depth,
                                              const extremz_params* params,
                                              extremz_report* report, void* stream);

/* EXTREMZ_NOALLOC_MAX_VOXELS of the loaded library. */
long long extremz_noalloc_max_voxels(void);

/* The critical-point lookup table in the layout of the reference's
 * src/LUT.bin (24 800 int32, read by loadLUTToGPU, src/ExtreM_cuda.cu:244-260).
 * Returns the number of entries written or -1. */
int extremz_lut(int32_t* out, int n);

const char* extremz_status_string(int status);
const char* extremz_last_cuda_error(void);

#ifdef __cplusplus
}
#endif

#endif /* EXTREMZ_H */
