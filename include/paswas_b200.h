/*
 * paswas_b200.h -- C ABI of the B200 Smith-Waterman engine (libpaswas_b200.so).
 *
 * Drop-in for the device side of pyPaSWAS's CUDA backend
 * (pyPaSWAS/Core/SmithWatermanCuda.py).  Plain pointers and sizes only; every
 * call returns a status code (PW_OK == 0, negative on error) and never aborts.
 * A human-readable message for the last failure is available from
 * pw_last_error().  One engine per host thread; calls on one engine are
 * serialised on its own CUDA stream.
 *
 * Host arrays are borrowed for the duration of a call.  Device memory is owned
 * by the engine.  Results stay valid until the next pw_align() or pw_destroy().
 */
#ifndef PASWAS_B200_H
#define PASWAS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; the Python layer maps them onto the reference's exceptions
 * (pyPaSWAS/Core/Exceptions.py): ARG -> InvalidOptionException,
 * DEVICE -> HardwareException, KERNEL/NOMEM/CAPACITY -> CudaException. */
#define PW_OK 0
#define PW_ERR_ARG (-1)
#define PW_ERR_DEVICE (-2)
#define PW_ERR_KERNEL (-3)
#define PW_ERR_NOMEM (-4)
#define PW_ERR_CAPACITY (-5)
#define PW_ERR_STATE (-6)
#define PW_ERR_TIMEOUT (-7)

/* pw_align() flags */
#define PW_FLAG_SCORE_ONLY 1u /* pair maxima only: no starting points, no walk */
#define PW_FLAG_PLAIN 2u      /* the unbatched form: one (query, target) pair per launch, as the reference
                                 launches one pair's kernels at a time; with integer scores each pair runs
                                 on the single-pair wavefront kernel (a warp per 256-row band), with fp32
                                 scores on one lane of the inter-sequence sweep */
#define PW_FLAG_INT32 4u      /* keep the score sweep on 32-bit lanes (no 16-bit dual-pair sweep) */
#define PW_FLAG_NO_CHAIN 8u   /* 16-bit sweep: run each multi-strip item on one warp (no chained strips) */
#define PW_FLAG_REPLAN 16u    /* rebuild the score sweep's work list even when inputs are unchanged */

typedef struct pw_engine pw_engine;

/* One alignment produced by the walk of SmithWaterman._print_alignments
 * (pyPaSWAS/Core/SmithWaterman.py:703-838).  Coordinates follow the
 * reference: s_* are query (x axis) positions, t_* target (y axis) positions,
 * both inclusive and 0-based.  The three alignment strings of the hit are
 * n_cols bytes each at strbuf + str_offset (sequence_match), + n_cols
 * (alignment), + 2 * n_cols (target_match). */
typedef struct {
    int32_t query;      /* index into the query list given to pw_set_queries */
    int32_t target;     /* index into the target list given to pw_set_targets */
    int32_t s_start, s_end, t_start, t_end;
    float score;        /* starting-point score (fp32, as the reference) */
    int32_t matches, mismatches;
    int32_t n_cols;
    int64_t str_offset;
} pw_hit;

typedef struct {
    int64_t pairs;          /* query x target pairs aligned */
    int64_t cells;          /* sum of len(q) * len(t) over the pairs */
    int64_t traced_pairs;   /* pairs swept for starting points (maximum reaches the start threshold) */
    int64_t minimum_pairs;  /* pairs whose maximum reached MINIMUM_SCORE */
    int64_t starting_points;
    int64_t hits;           /* hits kept by the walk (before the Python filter) */
    int64_t string_bytes;   /* bytes needed for all hit strings (3 * n_cols summed) */
    int32_t kernel_launches; /* launches of this library's kernels (library sorts and scans not counted) */
    int32_t truncated;      /* 1 when the starting-point cap cut the walk short */
    double score_ms, trace_ms, walk_ms; /* device time of the three phases */
    double score_kernel_ms; /* summed duration of the score-sweep launches */
    double trace_kernel_ms; /* summed duration of the direction-sweep launches */
    int32_t score_launches, trace_launches;
    int32_t orientation;    /* score sweep lanes: 0 = queries, 1 = targets */
    int32_t trace_orientation; /* direction sweep lanes: 0 = queries, 1 = targets */
    int64_t overflow_pairs; /* pairs recomputed on 32-bit lanes after reaching the 16-bit limit */
    int64_t traced_cells;   /* sum of len(q) * len(t) over the traced pairs */
    int64_t warp_pairs;     /* traced pairs swept one pair per warp (long targets) */
    int64_t cand_overflow_pairs; /* traced pairs swept twice: more candidates than the first slot held */
    double setup_ms;        /* host wall time between the phases: pruning, work lists, memory waves */
    double finish_ms;       /* host wall time after the device work: hit order, alignment strings */
    double total_ms;        /* host wall time of the whole call */
    int32_t score_path;     /* score sweep used: 0 16-bit strips, 1 32-bit / fp32 strips, 2 bands (pw_set_pairs
                               or few long sequences), 3 bands one pair per launch (PW_FLAG_PLAIN) */
    int32_t dual_lanes;     /* 16-bit score sweep in the dual-lane form: each strip against two lane
                               sequences per lane (1) instead of two strips against one (0) */
    int32_t waves;          /* memory waves of the direction sweep (0 when no pair was traced) */
    int32_t reuse;          /* work this call skipped because its inputs were unchanged since the last
                               call: PW_REUSE_QUERIES / PW_REUSE_TARGETS (the device copy and encodings of
                               that sequence set were kept), PW_REUSE_PLAN (the score sweep's work list
                               was kept) */
    int64_t h2d_bytes;      /* bytes this call copied host -> device (sequences, encodings, work lists) */
    int64_t d2h_bytes;      /* bytes this call copied device -> host (maxima, pair lists, starts, hits) */
    int32_t trace_store;    /* direction sweeps stored 1: each cell's 16-bit H, 0: 4-bit cell codes */
    int32_t tile_pairs;     /* traced long pairs in the tile form (checkpoints, tiles recomputed on the walk) */
    int64_t paired_cells;   /* cells of explicit pairs swept two to a warp in 16-bit halves (band16) */
} pw_run_info;

#define PW_REUSE_QUERIES 1
#define PW_REUSE_TARGETS 2
#define PW_REUSE_PLAN 4

/* Creates an engine on CUDA device `device`.
 * Replaces SmithWatermanCuda._initialize_device (SmithWatermanCuda.py:46-62). */
int pw_create(int device, pw_engine** out);

/* Releases all device memory of the engine (SmithWatermanCuda._clear_memory,
 * SmithWatermanCuda.py:69-94, plus the context pop of __del__, :40-43). */
void pw_destroy(pw_engine* e);

/* Message of the last failure on this engine ("" when none). */
const char* pw_last_error(pw_engine* e);

/* Free device memory in bytes (SmithWatermanCuda._device_global_mem_size,
 * SmithWatermanCuda.py:64-66). */
int pw_device_free_memory(pw_engine* e, int64_t* free_bytes, int64_t* total_bytes);

/* Scoring model and kernel constants.  Replaces the template substitution of
 * PaSWAS.Code.set_score_code (pyPaSWAS/Core/PaSWAS.py:55-72) and the per-shape
 * recompile of SmithWatermanCuda._compile_code (SmithWatermanCuda.py:170-174):
 * the engine takes these at run time.
 *   matrix        dim * dim substitution scores, row = query residue,
 *                 column = target residue, both minus char_offset
 *                 (default_score.cu:23, default_main.cu:234)
 *   gap, ext      gapScore / gapExtension; affine != 0 selects
 *                 calculateScoreAffineGap (SmithWaterman.py:149)
 *   lower_limit   LOWER_LIMIT_SCORE, minimum_score MINIMUM_SCORE, both fp32
 *                 as compiled (default_score.cu, default_main.cu:596,609)
 *   host_minimum  settings.minimum_score as the Python float the host walk
 *                 compares against (SmithWaterman.py:758)
 *   highest, filter_factor   give maxPossibleScore per pair,
 *                 fp32(highest * min(len_q, len_t) * filter_factor) evaluated
 *                 in double (SmithWatermanCuda.py:269-275)
 * Gap penalties must be <= 0. */
int pw_set_scoring(pw_engine* e, const float* matrix, int dim, int char_offset, float gap, float ext, int affine,
                   float lower_limit, float minimum_score, double host_minimum, double highest,
                   double filter_factor);

/* Query sequences (the x axis; records_seqs of SmithWaterman.align_sequences,
 * SmithWaterman.py:441).  residues: all sequences concatenated, unpadded,
 * upper-cased (the engine upper-cases ASCII letters itself; other bytes are
 * kept as given); offsets: n + 1 entries.  id_keys: one int per record, equal for
 * records whose ids are equal (same-id pairs are skipped,
 * SmithWaterman.py:752-755).  Replaces the query half of copy_sequences
 * (SmithWatermanCuda.py:176-184). */
int pw_set_queries(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                   const int32_t* id_keys);

/* Target sequences (the y axis), same conventions; they stay resident on the
 * device until replaced.  Replaces set_targets + the target half of
 * copy_sequences (SmithWaterman.py:370-414, SmithWatermanCuda.py:176-184). */
int pw_set_targets(pw_engine* e, const uint8_t* residues, const int64_t* offsets, int32_t n,
                   const int32_t* id_keys);

/* Aligns every query against every target: score sweep, starting-point
 * collection and the traceback walk.  Replaces SmithWaterman._calculate_score,
 * _traceback_host and the walk of _print_alignments (SmithWaterman.py:592-841)
 * with the kernel calls of SmithWatermanCuda._execute_calculate_score_kernel /
 * _execute_traceback_kernel (SmithWatermanCuda.py:191-259).
 * start_cap < 0: no cap; otherwise at most start_cap starting points are
 * walked, chosen in emission order (SmithWaterman.py:683-685). */
int pw_align(pw_engine* e, uint32_t flags, int64_t start_cap, pw_run_info* info);

/* Restricts pw_align to explicit (query, target) pairs instead of every query
 * against every target; n = 0 restores all-vs-all.  Indices refer to the
 * lists of pw_set_queries / pw_set_targets (checked by pw_align).  The
 * reference always aligns all-vs-all (SmithWaterman.align_sequences,
 * SmithWaterman.py:441-560); a caller who runs it once per pair, one query
 * and one target file each, gets exactly the hits of these pairs.  With
 * integer scores every listed pair is swept one warp per 256-row band, the
 * bands of a pair chained across warps (long pairs use the whole GPU).
 * pw_get_pair_max then holds -1 for the pairs that are not listed. */
int pw_set_pairs(pw_engine* e, const int32_t* query_idx, const int32_t* target_idx, int64_t n);

/* Queries whose hits are wanted: mask[q] != 0 traces query q's pairs as
 * usual; a 0 leaves its pairs at their maxima (pw_get_pair_max) and gives
 * them no starting points or hits, as if no cell reached the threshold.  n is
 * the number of queries of the last pw_set_queries, or 0 for no mask (every
 * query traced).  pw_set_queries clears the mask.  No counterpart in the
 * reference: the serving loop batches score-only and traceback requests in
 * one pw_align with it. */
int pw_set_query_trace(pw_engine* e, const uint8_t* mask, int32_t n);

/* Upper bound, in bytes, on the direction-matrix memory of one memory wave of
 * pw_align (4-bit cell codes -- direction, stop flag, candidate flag -- and a
 * 1-bit mark plane: half a byte plus one bit per traced cell); 0 restores the automatic choice (55% of the free
 * device memory with the candidate slots counted, at most 100 GiB).  Traced
 * pairs beyond the bound run in
 * further waves; a single pair larger than the bound runs alone.  Replaces
 * the batch sizing of SmithWaterman._get_max_number_sequences
 * (SmithWaterman.py:202-221) with its memory fraction `maximum_memory_usage`
 * (SmithWaterman.py:420-432). */
int pw_set_wave_limit(pw_engine* e, int64_t bytes);

/* Tuning knobs of the kernels' launch shapes and waits (no counterpart in the
 * reference, whose shapes are fixed template constants, default_main.cu:7-30).
 * Values 0 restore the automatic choice.
 *   PW_TUNE_CHAIN_MIN   16-bit score sweep: multi-strip items whose cost
 *                       reaches this many thousandths of the mean per-warp
 *                       load are cut into chained one-strip entries (default
 *                       500; 1 chains nearly every multi-strip item) */
#define PW_TUNE_CHAIN_MIN 0
/*   PW_TUNE_GRID_SHARE  thousandths of the GPU's resident-block capacity this
 *                       engine's persistent kernels may occupy (default all);
 *                       several engines (the serving loop's workers) can then
 *                       keep kernels resident side by side */
#define PW_TUNE_GRID_SHARE 1
/*   PW_TUNE_SEGMENT     chained 16-bit score sweep: queue entries per launch
 *                       (default all in one); shorter launches let other
 *                       engines' kernels in between (the serving loop) */
#define PW_TUNE_SEGMENT 2
/*   PW_TUNE_DUAL        16-bit score sweep form: 1 always dual lanes (one strip
 *                       against two lane sequences per lane), 2 never (two
 *                       strips against one lane sequence), 0 the cheaper of the
 *                       two by the cell-slot cost model (dual lanes win when
 *                       few sequences sit on the strip side, e.g. one query) */
#define PW_TUNE_DUAL 3
/*   PW_TUNE_CAND_SLOT   starting-point candidates held per traced pair before
 *                       its sweep is repeated with an exact slot (default
 *                       64); a small value exercises the repeat path */
#define PW_TUNE_CAND_SLOT 4
/*   PW_TUNE_WAIT_NS     longest wait, in nanoseconds, of a chained strip or
 *                       band for its predecessor's progress before the launch
 *                       gives up and pw_align fails with PW_ERR_KERNEL
 *                       (default 2,000,000,000) */
#define PW_TUNE_WAIT_NS 5
/*   PW_TUNE_STALL_TEST  1: the next chained launch makes one queue entry wait
 *                       on a progress flag that nothing sets, so that its wait
 *                       runs out (PW_TUNE_WAIT_NS) and pw_align reports the
 *                       failure; a test of the bounded waits.  0: off */
#define PW_TUNE_STALL_TEST 6
/*   PW_TUNE_LANES       score sweep lane width: 32 runs it on 32-bit lanes as
 *                       PW_FLAG_INT32 does; 0 the 16x2 sweep wherever the
 *                       scores allow it (pairs that reach the 16-bit limit are
 *                       recomputed on 32-bit lanes either way) */
#define PW_TUNE_LANES 7
/*   PW_TUNE_TRACE_STORE direction sweeps of linear integer scoring: 0 the
 *                       engine's choice (16-bit H per cell, cell codes derived
 *                       on read, when every traced maximum is below 2^15 and
 *                       the strip sweep holds most traced cells), 1 always
 *                       4-bit cell codes, 2 the H store wherever the maxima
 *                       allow it (the band sweep's long pairs included) */
#define PW_TUNE_TRACE_STORE 8
/*   PW_TUNE_TILE_TRACE  long pairs (the band sweep) of linear integer scoring:
 *                       0 the engine's choice (the tile form: a checkpoint
 *                       sweep, then 256 x 128-cell tiles of codes recomputed
 *                       where the walks need them), 1 the direction sweep's
 *                       stored cell codes (or H, PW_TUNE_TRACE_STORE), 2 the
 *                       tile form */
#define PW_TUNE_TILE_TRACE 9
int pw_set_tuning(pw_engine* e, int key, int64_t value);

/* Pair maxima (the last block of the maxima chain, default_main.cu:591),
 * row-major [n_queries][n_targets]. */
int pw_get_pair_max(pw_engine* e, float* out, int64_t n);

/* Hits of the last pw_align in the order the reference appends them to its
 * HitList: ascending score, then the pinned emission order of their starting
 * points.  strbuf receives the alignment strings (info->string_bytes); a null
 * strbuf copies the hit records only. */
int pw_get_hits(pw_engine* e, pw_hit* hits, int64_t max_hits, char* strbuf, int64_t strbuf_bytes);

/* The same records and strings without a copy: pointers into the engine's own
 * host copies, valid until the next pw_align, pw_set_* or pw_destroy on this
 * engine (the driver turns them into its Hit objects at once). */
int pw_get_hits_view(pw_engine* e, const pw_hit** hits, int64_t* n_hits, const char** strbuf, int64_t* strbuf_bytes);

/* Starting points of the last pw_align (StartingPoint layout of
 * default_main.cu:66-76, 36 bytes each) in emission order; `sequence` and
 * `target` are query / target list indices. */
int pw_get_starting_points(pw_engine* e, void* out36, int64_t max_points, int64_t* n_points);

/* Number of this library's kernels launched by the last pw_align. */
int pw_last_launch_count(pw_engine* e, int64_t* n);

/* Measurement helper (no counterpart in the reference): runs issue-rate
 * probes of the DPX add-max instructions the recurrences use and reports the
 * device's integer operation rates, counting each add and each max as one
 * operation: ops32 for __viaddmax_s32 (32-bit lanes), ops16x2 for
 * __viaddmax_s16x2 (two 16-bit lanes per instruction).  Used as the roofline
 * denominators by bench.py. */
int pw_measure_int_peak(pw_engine* e, double* ops32, double* ops16x2, double* ms);

/* ------------------------------------------------------------------------
 * Serving loop (no counterpart in the reference, which aligns one batch per
 * process): continuous batching of single-query requests against a database
 * kept resident on the device.
 *
 * W worker threads each own an engine (one CUDA stream) holding the database.
 * A worker that becomes free takes the requests waiting at that moment -- up to
 * max_batch of one mode, oldest first -- and runs them as one pw_align; the
 * batches of different workers overlap on the device.  Traceback requests are
 * admitted by direction-matrix memory: each reserves an estimate of its cell
 * codes (query length x database residues x the traced fraction seen so far,
 * at least 16 MiB) from `direction_budget` bytes shared by all workers; a
 * batch starts only when its reservation fits, and the engine's memory waves
 * (pw_set_wave_limit) keep its cell codes within it.  Every result equals that
 * of a lone pw_align of the query against the database.
 * ---------------------------------------------------------------------- */
#define PW_SERVE_TOP 0        /* pair maxima only; the top_k targets by maximum (ties: lower index) */
#define PW_SERVE_TRACEBACK 1  /* full path: the walk's hits of the query, in HitList order */

typedef struct pw_server pw_server;

typedef struct {
    int32_t status;          /* PW_OK or the failure of the request's batch */
    int32_t mode;
    int32_t batch_queries;   /* requests in the batch that carried this one */
    int32_t worker;
    int64_t cells;           /* len(query) x database residues */
    int64_t n_hits;          /* top hits (PW_SERVE_TOP) or walk hits (PW_SERVE_TRACEBACK) */
    int64_t string_bytes;    /* alignment strings of the hits */
    int64_t reserved_bytes;  /* direction-matrix reservation of the batch */
    double queue_ms;         /* submit -> batch start */
    double run_ms;           /* batch start -> result */
    double latency_ms;       /* submit -> result */
    double batch_score_kernel_ms; /* the batch's pw_run_info: score-sweep kernel time */
    double batch_setup_ms;   /* ... host planning time */
    double batch_call_ms;    /* ... whole pw_align call */
} pw_request_info;

typedef struct {
    int64_t submitted, completed, batches, cells, pending;
    int64_t budget_bytes, reserved_bytes, peak_reserved_bytes;
    double busy_ms;          /* summed wall time of the workers' batches */
    double traced_fraction;  /* current estimate used for reservations */
} pw_server_counters;

/* n_workers 1..16, max_batch 1..4096; direction_budget 0 = 8 GiB. */
int pw_server_create(int device, int n_workers, int max_batch, int64_t direction_budget, pw_server** out);
/* Finishes the waiting requests, then stops the workers and frees everything. */
void pw_server_destroy(pw_server* s);
const char* pw_server_last_error(pw_server* s);
/* Same arguments as pw_set_scoring; before pw_server_load_db. */
int pw_server_set_scoring(pw_server* s, const float* matrix, int dim, int char_offset, float gap, float ext,
                          int affine, float lower_limit, float minimum_score, double host_minimum, double highest,
                          double filter_factor);
/* The resident database (targets); id keys must be >= 0.  Once. */
int pw_server_load_db(pw_server* s, const uint8_t* residues, const int64_t* offsets, int32_t n,
                      const int32_t* id_keys);
/* Queues one query; returns at once with a ticket. */
int pw_server_submit(pw_server* s, const uint8_t* residues, int64_t length, int32_t mode, int32_t top_k,
                     int64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit; PW_ERR_TIMEOUT when it runs out). */
int pw_server_wait(pw_server* s, int64_t ticket, int32_t timeout_ms, pw_request_info* info);
/* Results of a finished request; buffers sized from pw_request_info. */
int pw_server_top_hits(pw_server* s, int64_t ticket, int32_t* targets, float* scores, int32_t k);
int pw_server_hits(pw_server* s, int64_t ticket, pw_hit* hits, int64_t max_hits, char* strbuf,
                   int64_t strbuf_bytes);
/* pw_set_tuning on every worker engine, or, for the keys below, a setting of
 * the server's own scheduler:
 *   PW_SERVE_TUNE_POLICY   0: batches in arrival order; 1 (default): the
 *                          shortest waiting queries first, except that a
 *                          request waiting longer than PW_SERVE_TUNE_AGE_MS
 *                          goes first (no request starves)
 *   PW_SERVE_TUNE_AGE_MS   the waiting time after which policy 1 serves a
 *                          request in arrival order (default 25)
 *   PW_SERVE_TUNE_MAX_BATCH  requests per batch (as at pw_server_create)
 *   PW_SERVE_TUNE_MAX_RESIDUES  query residues per batch (0: no limit): a
 *                          batch's requests all finish when it does, so this
 *                          bounds the run time a request can wait for; the
 *                          first request of a batch always joins */
#define PW_SERVE_TUNE_POLICY 100
#define PW_SERVE_TUNE_AGE_MS 101
#define PW_SERVE_TUNE_MAX_BATCH 102
#define PW_SERVE_TUNE_MAX_RESIDUES 103
int pw_server_tune(pw_server* s, int key, int64_t value);
/* Frees a finished request's results. */
int pw_server_release(pw_server* s, int64_t ticket);
int pw_server_stats(pw_server* s, pw_server_counters* st);

/* Pair maxima without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc themselves or have
 * the library do it -- code running where another component owns all device
 * memory (a framework's caching allocator, a fixed serving budget), or a
 * latency-critical path where cudaMalloc's implicit device synchronisation
 * is not acceptable.
 *
 * Same result as pw_align() with PW_FLAG_SCORE_ONLY followed by
 * pw_get_pair_max(): every query (x axis) against every target (y axis),
 * pair_max[q * nt + t], host buffers in and out, no engine needed.  Scoring
 * arguments are those of pw_set_scoring().  All device working memory is one
 * 64 MiB array inside the library that every GPU loading the library keeps
 * until the process exits; inputs whose staged size (sequences, work list,
 * results and the boundary rows of targets longer than one strip) exceeds it
 * are rejected with PW_ERR_CAPACITY and a message in err.  Calls share that
 * array: the library serialises them with a host lock, and their GPU work must
 * not overlap with other users of it.  The first call on a device looks up the
 * array's device address (make it before any stream capture on that device).
 * Runs on the legacy default stream and returns when pair_max is filled; the
 * calling thread's current device is the same on return as on entry. */
int pw_score_max_noalloc(int device, const float* matrix, int dim, int char_offset, float gap, float ext,
                         int affine, const uint8_t* q_residues, const int64_t* q_offsets, int32_t n_queries,
                         const uint8_t* t_residues, const int64_t* t_offsets, int32_t n_targets, float* pair_max,
                         char* err, int32_t err_bytes);

/* ---------------------------------------------------------------------------
 * trimmedFasta output without Python Hit objects (host only, no device).
 * Replaces, for the trimmer's output, the chain Hit construction
 * (SmithWaterman._print_alignments, SmithWaterman.py:822-838) -> _filter_hit
 * (:843-848) -> HitList.append (HitList.py:28-52) -> TrimmerFormatter
 * (Formatters.py:110-150, Hit.get_trimmed_line, Hit.py:274-286), byte for
 * byte.  `hits` are pw_get_hits records in walk order, their query / target
 * indices below n_queries / n_targets.  Per query q: q_rank[q] the rank of its id in Python's string order
 * (equal ids, equal ranks), its original length and start position, its id
 * bytes q_id[q_id_off[q] .. q_id_off[q + 1]) and its sequence as given
 * q_seq[q_seq_off[q] ..) (ASCII).  Per target: the same, t_id with the "_RC"
 * suffix already removed as the formatter removes it.  thresholds: relative
 * score, query identity, query coverage, base score.  With out == NULL the
 * call only stores the byte count in *out_len; otherwise it writes the
 * records (each ">target query\n trimmed query \n") and fails with
 * PW_ERR_CAPACITY when out_cap is too small.  An invalid hit location returns
 * PW_ERR_ARG (the reference raises there). */
int pw_trimmed_fasta(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                     const int32_t* q_rank, const int64_t* q_orig_len,
                     const int64_t* q_start_pos, const char* q_id, const int64_t* q_id_off, const char* q_seq,
                     const int64_t* q_seq_off, const int32_t* t_rank, const int64_t* t_orig_len,
                     const int64_t* t_start_pos, const char* t_id, const int64_t* t_id_off, const double* thresholds,
                     char* out, int64_t out_cap, int64_t* out_len);

/* TXT output (DefaultFormatter, Formatters.py:3-47) of the same HitList, byte
 * for byte, Python's float repr included: per record the summary line and the
 * three alignment strings, each line ending in a newline.  Arguments as
 * pw_trimmed_fasta's, plus strbuf / strbuf_bytes (the pw_get_hits strings)
 * and without the query sequences; t_id holds the target ids as they are. */
int pw_txt_records(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                   const char* strbuf, int64_t strbuf_bytes,
                   const int32_t* q_rank, const int64_t* q_orig_len, const int64_t* q_start_pos, const char* q_id,
                   const int64_t* q_id_off, const int32_t* t_rank, const int64_t* t_orig_len,
                   const int64_t* t_start_pos, const char* t_id, const int64_t* t_id_off, const double* thresholds,
                   char* out, int64_t out_cap, int64_t* out_len);

/* SAM output (SamFormatter, Formatters.py:51-106; Hit.get_sam_line and
 * get_sam_sq, Hit.py:222-272,298-304,338-406) of the same HitList, byte for
 * byte: "@HD", the "@SQ" lines, "@PG", one alignment line per hit (CIGAR,
 * RC flag and mirroring, reverse-complemented SEQ, AS/RS/BS/QC/QI fields with
 * Python's float repr).  Arguments as pw_txt_records's plus the query
 * sequences (q_seq / q_seq_off, as pw_trimmed_fasta takes them); q_id and
 * t_id hold the ids as they are. */
int pw_sam_records(const pw_hit* hits, int64_t n_hits, int32_t n_queries, int32_t n_targets,
                   const char* strbuf, int64_t strbuf_bytes, const int32_t* q_rank, const int64_t* q_orig_len,
                   const int64_t* q_start_pos, const char* q_id, const int64_t* q_id_off, const char* q_seq,
                   const int64_t* q_seq_off, const int32_t* t_rank, const int64_t* t_orig_len,
                   const int64_t* t_start_pos, const char* t_id, const int64_t* t_id_off, const double* thresholds,
                   char* out, int64_t out_cap, int64_t* out_len);

/* ---------------------------------------------------------------------------
 * Sequence records read natively (host only, no device).  Replaces the
 * reference's record preparation for the engine: BioPythonReader.read_records
 * (pyPaSWAS/Core/Readers.py:90-118; Biopython's FASTA / FASTQ parsing, the
 * islice(start, end) of the file's records, the limit_length filter that keeps
 * 0 < len <= limit_length when limit_length > 0, SWSeqRecord's upper-casing,
 * SWSeqRecord.py:16), the target transforms complement_records,
 * complement_records_only and reverse_records (Readers.py:68-86, ids + "_RC")
 * and sort_records (Readers.py:30-34: stable, longest first), as
 * Pypaswas._get_query_sequences / _get_target_sequences chain them
 * (pypaswasall.py:98-124).  The records come out packed: residues with
 * offsets (n + 1) and ids with offsets (n + 1), in the final order. */
#define PW_FORMAT_FASTA 0
#define PW_FORMAT_FASTQ 1
#define PW_RECORDS_AS_READ 0        /* queries, and targets of non-DNA scores */
#define PW_RECORDS_APPEND_RC 1      /* complement_records: + reverse complements */
#define PW_RECORDS_RC_ONLY 2        /* complement_records_only: the reverse complements alone */
#define PW_RECORDS_APPEND_REVERSED 3 /* reverse_records: + reversed copies */
typedef struct pw_records pw_records;
/* Parses `bytes` of FASTA / FASTQ text; end < 0 reads to the last record, an
 * end before start selects no record (as islice does).
 * Malformed FASTQ fails with PW_ERR_ARG and a message in err. */
int pw_records_parse(const char* data, int64_t bytes, int format, int64_t start, int64_t end, int64_t limit_length,
                     int transform, int sort_desc, pw_records** out, char* err, int32_t err_bytes);
/* The same on a file (BioPythonReader's path argument). */
int pw_records_read(const char* path, int format, int64_t start, int64_t end, int64_t limit_length, int transform,
                    int sort_desc, pw_records** out, char* err, int32_t err_bytes);
/* Record count, residue bytes, id bytes and the records the length limit removed. */
int pw_records_sizes(const pw_records* r, int64_t* n_records, int64_t* residue_bytes, int64_t* id_bytes,
                     int64_t* dropped);
/* Copies the packed records into caller buffers sized from pw_records_sizes. */
int pw_records_copy(const pw_records* r, uint8_t* residues, int64_t* offsets, char* ids, int64_t* id_offsets);
void pw_records_free(pw_records* r);
/* Dense ranks of n byte strings blob[off[i], off[i + 1]) in byte order (a
 * prefix before its extensions; equal strings share a rank): Python's string
 * order of ASCII record ids, which HitList de-duplication and the formatters'
 * (query id, target id, score) sort compare (HitList.py:28-52,
 * Formatters.py:34-37).  The formatters take these ranks (pw_trimmed_fasta,
 * pw_txt_records). */
int pw_id_ranks(const char* blob, const int64_t* off, int64_t n, int32_t* ranks);

#ifdef __cplusplus
}
#endif
#endif
