/*
 * blastp_b200.h -- native C ABI of the B200 blastp preliminary-search engine:
 * two-hit word finding + BLOSUM62 X-drop ungapped extension.
 *
 * Everything here is extern "C", plain pointers and sizes.  The reference's
 * own entry points (GPU_BLASTP and family) are declared in
 * gpu_cpu_common_b200.h and implemented on top of this engine.
 *
 * Reference interfaces replaced (file:line into avtomaton/blastp-cuda):
 *   bp_search            GPU_BLASTP + GPU_BLASTP_get_data
 *                        (gpu_blastp.cu:16-259, ncbi_blast_files/gpu_cpu_common.h:44-69),
 *                        returning the full HSP set instead of 2 slots per subject
 *   bp_query_create      the NCBI-built lookup table it consumes
 *                        (BlastAaLookupTable, read at gpu_blastp.cu:45-61)
 *   bp_db_create         the .gpu volume upload (gpu_blastp.cu:139-163,
 *                        ncbi_blast_files/functions.cpp:620-699)
 *   bp_hsp               GPUBlastInitHitList (ncbi_blast_files/gpu_cpu_common.h:29-38)
 *   counters             d_Hits[oid*3+{0,1,2}] (gpu_blastp_kernel.cu:310-312)
 *
 * Status codes replace the reference's void returns; no call falls back to
 * the CPU.  Device memory is owned by the handles; host buffers by the caller.
 */
#ifndef BLASTP_B200_H
#define BLASTP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bp_status {
    BP_OK = 0,
    BP_ERR_INVALID = 1,       /* bad argument (size, residue code, parameter) */
    BP_ERR_CUDA = 2,          /* a CUDA runtime call failed; see bp_last_error() */
    BP_ERR_NOMEM = 3,         /* device allocation failed */
    BP_ERR_TOO_LARGE = 4,     /* input beyond a stated limit */
    BP_ERR_TIMEOUT = 5,       /* a bounded device wait ran out */
    BP_ERR_NOT_READY = 6,     /* asynchronous work still in flight */
    BP_ERR_NO_DEVICE = 7      /* no CUDA device visible */
} bp_status;

/* Search parameters.  Defaults (bp_params_default): word 3, T 11, window 40,
 * x_dropoff 16 raw (7 bits at lambda_u 0.3176), cutoff_score 41 raw. */
typedef struct bp_params {
    int32_t word_length;      /* must be 3 */
    int32_t threshold;        /* neighbour-word score threshold T */
    int32_t window;           /* two-hit window */
    int32_t x_dropoff;        /* raw X-drop for ungapped extension */
    int32_t cutoff_score;     /* raw score an HSP must reach to be reported */
} bp_params;

/* One ungapped HSP; same layout and meaning as GPUBlastInitHitList. */
typedef struct bp_hsp {
    int32_t hsp_q;            /* query start of the HSP */
    int32_t hsp_s;            /* subject start of the HSP */
    int32_t query_offset;     /* query offset of the second word hit */
    int32_t subject_offset;   /* subject offset of the second word hit */
    int32_t hsp_len;          /* HSP length */
    int32_t score;            /* raw ungapped score */
} bp_hsp;

typedef struct bp_engine bp_engine;   /* device, stream, scratch */
typedef struct bp_db bp_db;           /* HBM-resident subject database */
typedef struct bp_query bp_query;     /* device query + neighbour-word table */
typedef struct bp_result bp_result;   /* device counters + HSP CSR */

/* Limits. */
#define BP_MAX_QUERY_LENGTH 65535     /* query offsets are stored as uint16 */
#define BP_ALPHABET 28                /* NCBIstdaa; residue codes 0..27 */

void bp_params_default(bp_params* p);
const char* bp_status_string(bp_status s);

/* Host-side copy of the int8 28x28 BLOSUM62 (NCBIstdaa order) the engine
 * scores with.  Needs no GPU. */
void bp_blosum62_ncbistdaa(int8_t out[BP_ALPHABET * BP_ALPHABET]);

/* Engine: binds a CUDA device and creates a non-blocking stream. */
bp_status bp_engine_create(int device, bp_engine** out);
void bp_engine_destroy(bp_engine* e);
const char* bp_last_error(const bp_engine* e);
void* bp_engine_stream(bp_engine* e);               /* cudaStream_t */
uint64_t bp_engine_launch_count(const bp_engine* e); /* kernels launched so far */
float bp_engine_last_scan_ms(const bp_engine* e);    /* scan kernel time of the last search */
bp_status bp_engine_synchronize(bp_engine* e);
/* The longest a streaming bp_blastp_host call lets its scan wait for one
 * upload chunk to arrive (default 20,000 ms); past it the scan stops and the
 * call returns BP_ERR_TIMEOUT, leaving the engine usable.  No counterpart in
 * the reference, whose upload completes before its launch. */
bp_status bp_engine_set_upload_wait(bp_engine* e, uint32_t ms);
/* Fault injection for tests of that bounded wait: the next bp_blastp_host
 * call that streams copies upload chunk `chunk` but does not announce its
 * arrival, so the scan's wait for it runs out (chunk < 0: none). */
bp_status bp_engine_drop_chunk_flag(bp_engine* e, int32_t chunk);

/* Database: residues (NCBIstdaa, each < 28) of n_subjects subjects laid end
 * to end, with n_subjects+1 int64 offsets.  bp_db_create copies from host
 * memory (synchronously); bp_db_create_device copies from device memory. */
bp_status bp_db_create(bp_engine* e, const uint8_t* residues, int64_t n_residues,
                       const int64_t* offsets, int32_t n_subjects, bp_db** out);
bp_status bp_db_create_device(bp_engine* e, const uint8_t* d_residues, int64_t n_residues,
                              const int64_t* d_offsets, int32_t n_subjects, bp_db** out);
void bp_db_destroy(bp_db* db);
int32_t bp_db_subjects(const bp_db* db);
int64_t bp_db_residues(const bp_db* db);

/* Database file: the subjects on disk in volumes of at most volume_residues
 * residues (<= 0: 1 GiB), optionally stored longest first (an oid map then
 * gives every stored subject's original index).  Replaces the reference's
 * ".gpu" file (functions.cpp:364-613, 4 GB volume cap at :481-485).
 * bp_dbfile_info / bp_dbfile_read_host need no GPU; bp_db_open maps the file
 * and streams it into HBM through two pinned staging buffers, so the host
 * copy of one part overlaps the transfer of the previous one. */
bp_status bp_dbfile_write(const char* path, const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                          int32_t n_subjects, int64_t volume_residues, int32_t sort_by_length);
bp_status bp_dbfile_info(const char* path, int32_t* n_subjects, int64_t* n_residues, int32_t* n_volumes,
                         int32_t* sorted);
/* residues [n_residues], offsets [n_subjects+1] (stored order), oids
 * [n_subjects] (original index of each stored subject); any may be NULL. */
bp_status bp_dbfile_read_host(const char* path, uint8_t* residues, int64_t* offsets, int32_t* oids);
bp_status bp_db_open(bp_engine* e, const char* path, bp_db** out);

/* Query: copies the residues to the device and builds the neighbour-word
 * table there (CSR keyed by the packed 3-letter code, plus presence bitmap). */
bp_status bp_query_create(bp_engine* e, const uint8_t* residues, int32_t length,
                          const bp_params* params, bp_query** out);
void bp_query_destroy(bp_query* q);
/* Copies the table back: cell_start[32769] (uint32) and up to cap entries. */
bp_status bp_query_table(bp_query* q, uint32_t* cell_start, uint16_t* entries, int64_t cap,
                         int64_t* n_entries);

/* Plain search of one query against subjects [first, first+count) of db
 * (count < 0: to the end).  Enqueued on the engine stream; the result's
 * buffers are valid once bp_result_wait returns BP_OK. */
bp_status bp_search(bp_engine* e, const bp_db* db, const bp_query* q, int32_t first,
                    int32_t count, bp_result** out);
bp_status bp_result_wait(bp_result* r);
int32_t bp_result_subjects(const bp_result* r);
int64_t bp_result_hsps(const bp_result* r);          /* after bp_result_wait */
/* Copies results to host memory.  Any pointer may be NULL.
 *   counters  int32[3*subjects]: hits, successful extensions, extensions
 *   hsp_off   int64[subjects+1]: CSR offsets into hsps
 *   hsps      bp_hsp[bp_result_hsps()], per subject in discovery order */
bp_status bp_result_copy(bp_result* r, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps);
/* A 128-bit digest of the result (counters, CSR offsets, HSP records in
 * order), computed on the device; equal results give equal digests, and
 * different ones differ with overwhelming probability.  For comparing large
 * result sets without copying them to the host (bp_batch_digest and
 * bp_server_digest give the same digest for the same result).  No
 * counterpart in the reference. */
bp_status bp_result_digest(bp_result* r, uint64_t out[2]);
void bp_result_destroy(bp_result* r);

/* ---- Gapped stage: the consumer of the ungapped HSPs -------------------
 * Replaces the call the reference makes after ingesting the ungapped HSPs,
 * aux_struct->GetGappedScore (ncbi_blast_files/blast_engine.c:588-591), which
 * is NCBI BLAST+ code not shipped with the reference.  Score-only gapped
 * X-drop extension with affine gaps (Altschul et al. 1997), on the device,
 * from each ungapped HSP of a finished single-context search:
 *  - a subject's ungapped HSPs are taken by descending score (equal scores in
 *    discovery order); one whose query and subject ranges both lie inside a
 *    gapped HSP already reported for the subject is skipped;
 *  - seed: the middle letter of an HSP of at most 11 letters, else offset 5
 *    of its first highest-scoring 11-letter window;
 *  - two dynamic programmes from the seed: leftwards over the letters up to
 *    and including the seed pair, rightwards over the letters after it, each
 *    with H = max(diagonal + S, E, F), E/F = max(H - open, E/F) - extend
 *    (a k-letter gap costs open + k * extend), cells below the best score so
 *    far minus x_dropoff dead (tested once per query row, after the row), a
 *    row's band running from the previous row's first live column to one past
 *    its last, then on while the horizontal-gap score stays >= best -
 *    x_dropoff; each returns its best score and the first cell (lowest row,
 *    then column) reaching it;
 *  - the gapped HSP (score = left + right) is reported when score >=
 *    cutoff_score.
 * Defaults: open 11, extend 1 (BLOSUM62's usual costs), x_dropoff 38 (15
 * bits at the gapped lambda 0.267), cutoff 0. */
typedef struct bp_gapped bp_gapped;
typedef struct bp_gapped_params {
    int32_t gap_open;         /* 0..65535 */
    int32_t gap_extend;       /* 1..255 */
    int32_t x_dropoff;        /* raw, 0..2^20 */
    int32_t cutoff_score;     /* raw */
} bp_gapped_params;
typedef struct bp_gapped_hsp {
    int32_t score;
    int32_t q_start, q_end;   /* query range, end exclusive */
    int32_t s_start, s_end;   /* subject range, end exclusive */
    int32_t q_seed, s_seed;   /* the seed pair */
    int32_t ungapped;         /* the ungapped HSP it came from (index within its subject) */
} bp_gapped_hsp;
void bp_gapped_params_default(bp_gapped_params* p);
/* Runs the gapped stage on r (waits for it).  The search's database and
 * query must still exist.  Per subject out: counters {ungapped HSPs, gapped
 * HSPs reported, extensions run}, and the reported HSPs as CSR in processing
 * order.  Bands of up to 2,048 columns run in the main launch; a subject
 * with a wider band is redone by a second launch with a ring spanning it. */
bp_status bp_gapped_run(bp_result* r, const bp_gapped_params* p, bp_gapped** out);
/* The same with a given band ring width (a power of two >= 64), for tests of
 * the wide-band path. */
bp_status bp_gapped_run_ring(bp_result* r, const bp_gapped_params* p, int32_t ring_columns, bp_gapped** out);
int64_t bp_gapped_hsps(const bp_gapped* g);
float bp_gapped_ms(const bp_gapped* g);              /* device time of the stage */
/* Copies to host memory (any pointer may be NULL): counters int32[3*n],
 * off int64[n+1], hsps bp_gapped_hsp[bp_gapped_hsps()]. */
bp_status bp_gapped_copy(bp_gapped* g, int32_t* counters, int64_t* off, bp_gapped_hsp* hsps);
void bp_gapped_destroy(bp_gapped* g);

/* One call from host buffers to host buffers: uploads the database and the
 * query, searches, and copies the results back (the end-to-end form).
 * hsps may be NULL to only size the result (n_hsps out).  The upload runs
 * under the scan: from pinned residues (cudaMallocHost / cudaHostRegister)
 * one scan launch follows 8 MiB chunks as they arrive; from pageable memory
 * each chunk gets its own launch, and pinned counters receive each chunk's
 * counters as soon as its scan ends.  BP_ERR_INVALID for offsets out of order
 * or residue codes >= 28 (checked on the device); BP_ERR_TIMEOUT if a chunk
 * did not arrive within 20 s. */
bp_status bp_blastp_host(bp_engine* e, const uint8_t* query, int32_t qlen, const bp_params* p,
                         const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                         int32_t n_subjects, int32_t* counters, int64_t* hsp_off,
                         bp_hsp* hsps, int64_t hsp_cap, int64_t* n_hsps);

/* ---- batched search ------------------------------------------------------
 * Many queries against one resident database in one persistent launch.  The
 * reference runs one launch per query (gpu_blastp.cu:197-210); here the
 * subjects are cut into chunks of about chunk_residues residues and every
 * (query, chunk) pair is a work item.  Each query's results are identical to
 * its bp_search results. */
typedef struct bp_batch bp_batch;

typedef enum {
    BP_SCHED_DYNAMIC = 0,   /* CTAs take items from one global cursor */
    BP_SCHED_STATIC = 1,    /* item i goes to CTA i mod ctas */
    BP_SCHED_COSTS = 2,     /* longest predicted item first into the least loaded CTA */
    BP_SCHED_COST_ORDER = 3 /* one global cursor over the items, longest predicted first */
} bp_schedule;

typedef struct {
    int32_t chunk_residues;     /* residues per chunk (a chunk holds at least one subject) */
    int32_t schedule;           /* bp_schedule */
    int32_t ctas;               /* persistent CTAs (0: one per SM) */
    int32_t max_warps;          /* warps per CTA cap (0: as many as shared memory allows) */
    int32_t use_graph;          /* capture the launch sequence once, replay it on bp_batch_run */
    const float* item_costs;    /* BP_SCHED_COSTS, BP_SCHED_COST_ORDER: predicted cost of item q*n_chunks + c */
    int32_t subject_first;      /* subjects [subject_first, subject_first + subject_count) */
    int32_t subject_count;      /* (< 0: to the end of the database) */
    int32_t pack_residues;      /* > 0: queries of at most half this length share tables of up to
                                   this many offsets (32 queries at most), so one word scan of a
                                   subject serves all of them; 0: every query alone.
                                   Default 512. */
    int32_t plain_unpacked;     /* 1: every query that is not packed runs as the plain single-query
                                   scan over the batch's subjects (subject cursor, longest first),
                                   the packed tables as batched items; the item schedule then
                                   applies to the packed tables only.  Default 0. */
} bp_batch_options;

void bp_batch_options_default(bp_batch_options* o);
/* Chunk boundaries the batch would use over subjects [subject_first,
 * subject_first + subject_count) (count < 0: to the end): chunk c holds
 * subjects [chunk_first[c], chunk_first[c+1]).  chunk_first may be NULL to
 * only count. */
bp_status bp_batch_plan(const bp_db* db, int32_t subject_first, int32_t subject_count, int32_t chunk_residues,
                        int32_t* chunk_first, int32_t* n_chunks);
/* Creates the batch and enqueues its first run.  The engine, database and
 * queries must outlive the batch.  All queries share one window. */
bp_status bp_search_batch(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                          const bp_batch_options* opt, bp_batch** out);
/* Enqueues the same search again (a graph replay when use_graph is set). */
bp_status bp_batch_run(bp_batch* b);
bp_status bp_batch_wait(bp_batch* b);
int64_t bp_batch_hsps(const bp_batch* b);            /* all queries, after bp_batch_wait */
int32_t bp_batch_items(const bp_batch* b);
float bp_batch_last_scan_ms(const bp_batch* b);      /* device time of the last run's scan launch */
/* Query qi's results in the bp_result_copy layout (offsets start at 0),
 * for the batch's subjects (index 0 = subject_first). */
bp_status bp_batch_copy_query(bp_batch* b, int32_t qi, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                              int64_t* n_hsps);
/* Query qi's result digest (as bp_result_digest). */
bp_status bp_batch_digest(bp_batch* b, int32_t qi, uint64_t out[2]);
/* Predicted load of each CTA queue (BP_SCHED_COSTS), for reporting. */
bp_status bp_batch_queue_costs(const bp_batch* b, double* costs, int32_t* n_queues);
/* Queue (index into bp_batch_queue_costs' list) of every item q*n_chunks + c;
 * -1 under BP_SCHED_DYNAMIC. */
bp_status bp_batch_item_queues(const bp_batch* b, int32_t* queue_of_item);
void bp_batch_destroy(bp_batch* b);

/* ---- learned cost model ---------------------------------------------------
 * A two-layer MLP (ReLU hidden layer, fp32) that predicts each work item's
 * word-hit and extension counts, trained and evaluated on the device with
 * the library's own kernels.  No counterpart in the reference. */
typedef struct bp_mlp bp_mlp;
#define BP_COST_FEATURES 24

/* Residue counts per chunk (28 bins, NCBIstdaa codes), on the device. */
bp_status bp_db_chunk_histograms(bp_engine* e, const bp_db* db, const int32_t* chunk_first, int32_t n_chunks,
                                 uint32_t* counts);
/* Features of item q*n_chunks + c, BP_COST_FEATURES floats each:
 * log(1+query length), log(1+neighbour-word entries), log(1+chunk residues),
 * the chunk's composition over the 20 standard residues (fractions), and the
 * caller's planted-homolog density (0 when unknown). */
bp_status bp_batch_features(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                            const int32_t* chunk_first, int32_t n_chunks, float planted_density, float* X);
bp_status bp_mlp_create(bp_engine* e, int32_t n_in, int32_t n_hidden, int32_t n_out, uint64_t seed, bp_mlp** out);
void bp_mlp_destroy(bp_mlp* m);
int32_t bp_mlp_num_params(const bp_mlp* m);
/* Parameters W1[in][hidden], b1[hidden], W2[hidden][out], b2[out]; norm =
 * x_mean[in], x_std[in], y_mean[out], y_std[out].  Either may be NULL. */
bp_status bp_mlp_get_params(bp_mlp* m, float* params, float* norm);
bp_status bp_mlp_set_params(bp_mlp* m, const float* params, const float* norm);
/* Mean squared error over rows and outputs, and its gradient with respect to
 * the parameters, on raw inputs (no standardisation). */
bp_status bp_mlp_loss_grad(bp_mlp* m, const float* X, const float* T, int32_t n, float* loss, float* grad);
/* Standardises X and T per column (kept in the model), then trains with Adam
 * on shuffled minibatches.  loss_curve: optional, one value per epoch. */
bp_status bp_mlp_fit(bp_mlp* m, const float* X, const float* T, int32_t n, int32_t epochs, int32_t batch, float lr,
                     uint64_t seed, float* loss_curve);
bp_status bp_mlp_predict(bp_mlp* m, const float* X, int32_t n, float* Y);

/* Item costs for BP_SCHED_COSTS from a model predicting log(1 + hits) and
 * log(1 + extensions):  cost = w[0]*residues + w[1]*hits + w[2]*extensions. */
bp_status bp_batch_predict_costs(bp_engine* e, bp_mlp* model, const float* weights, const bp_db* db,
                                 const bp_query* const* queries, int32_t n_queries, const int32_t* chunk_first,
                                 int32_t n_chunks, float planted_density, float* costs);

/* ---- GPU/CPU co-scheduling -------------------------------------------------
 * Splits the subjects between the device ([0, split)) and a CPU search of
 * the rest so both finish together, from predicted device time per chunk and
 * the CPU's time per unit of device time (cpu_factor, measured by the
 * caller).  Replaces the reference's fixed GPU share of the OIDs
 * (functions.cpp:125-149, :1059).  bp_cosched_split_costs needs no GPU. */
int32_t bp_cosched_split_costs(const double* chunk_costs, int32_t n_chunks, double cpu_factor);
bp_status bp_cosched_split(bp_engine* e, bp_mlp* model, const float* weights, const bp_db* db,
                           const bp_query* const* queries, int32_t n_queries, float planted_density, double cpu_factor,
                           int32_t* split_subject);

/* ---- autotuner -------------------------------------------------------------
 * Times candidate batch configurations on the first sample_subjects subjects
 * with the whole query set and returns the fastest: first every subject-chunk
 * size with every packing size (dynamic schedule, all warps), then, at the
 * best of those, the other schedules and the warp caps, and last the best
 * one with plain_unpacked set. */
typedef struct {
    int32_t chunk_residues, schedule, max_warps;
    float ms;                   /* best scan time of the candidate on the sample */
    int32_t pack_residues;
    int32_t plain_unpacked;
} bp_autotune_trial;

typedef struct {
    const int32_t* chunk_sizes; /* NULL: 64Ki, 256Ki, 1Mi, 4Mi residues */
    int32_t n_chunk_sizes;
    const int32_t* warp_caps;   /* NULL: {0 (as many as fit), 16} */
    int32_t n_warp_caps;
    int32_t schedules_mask;     /* bit s tries bp_schedule s; BP_SCHED_COSTS needs model */
    bp_mlp* model;
    float cost_weights[3];
    float planted_density;
    int32_t sample_subjects;    /* <= 0: 1/16 of the database */
    int32_t reps;               /* timed runs per candidate, best kept */
    const int32_t* pack_sizes;  /* NULL: {0, 512, 1024} (bp_batch_options.pack_residues) */
    int32_t n_pack_sizes;
} bp_autotune_options;

void bp_autotune_options_default(bp_autotune_options* o);
bp_status bp_batch_autotune(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                            const bp_autotune_options* opt, bp_batch_options* best, bp_autotune_trial* trials,
                            int32_t trials_cap, int32_t* n_trials);

/* ---- serving ---------------------------------------------------------------
 * Continuous batching against one resident database.  Requests are admitted
 * in arrival order while the device-memory budget allows, and launched as
 * batched searches on free lanes (each lane: its own stream and scratch, a
 * 1/lanes share of the SMs), so a batch admitted while another runs
 * overlaps it.  A request's results stay on the device until it is
 * released.  No counterpart in the reference. */
typedef struct bp_server bp_server;

enum {
    BP_REQ_UNKNOWN = -1,
    BP_REQ_QUEUED = 0,
    BP_REQ_ADMITTED = 1,
    BP_REQ_RUNNING = 2,
    BP_REQ_DONE = 3,
    BP_REQ_FAILED = 4
};

typedef struct {
    int32_t max_batch_queries;      /* queries per launch */
    int64_t device_memory_budget;   /* bytes held by admitted requests */
    int32_t chunk_residues;
    int32_t schedule;               /* bp_schedule; BP_SCHED_COSTS uses model */
    int32_t lanes;                  /* batches in flight at once (1..16) */
    int32_t poll_us;                /* dispatcher poll interval */
    bp_mlp* model;                  /* used by the server's thread only while it exists */
    float cost_weights[3];
    float planted_density;
    bp_params params;
    int32_t lane_depth;             /* batches queued per lane (>= 1): a lane runs its batches one
                                       after the other on the device, in admission order, while the
                                       next ones are prepared and launched behind them */
    int32_t admission;              /* BP_ADMIT_ARRIVAL (default) or BP_ADMIT_SHORTEST: the shortest
                                       waiting query is admitted first (lower median latency under
                                       load, longer waits for long queries) */
    int32_t segments;               /* 1 (default): a request's search is one job over the whole
                                       database.  2..64: it runs as this many jobs over consecutive
                                       subject ranges of about equal residues, one query each, and
                                       every free slot takes the next range of the request chosen by
                                       `admission` -- arrival order, or (BP_ADMIT_SHORTEST) the least
                                       remaining work (ranges left x query length), so a short
                                       request that arrives while a long one runs goes ahead of the
                                       long one's remaining ranges.  max_batch_queries is not used;
                                       each range runs as the plain single-query search (as does,
                                       with one lane, any batch of one request).  Results are the
                                       same either way. */
    int32_t max_wait_ms;            /* BP_ADMIT_SHORTEST: a request that has waited this long since
                                       it arrived goes before shorter ones (oldest first), which
                                       bounds how long long requests starve; 0 (default): never */
} bp_server_options;

enum { BP_ADMIT_ARRIVAL = 0, BP_ADMIT_SHORTEST = 1 };

typedef struct {
    int64_t completed, failed, batches, pending;
    double mean_batch;
    int32_t max_in_flight;
    int64_t mem_used, mem_peak;
    double p50_ms, p99_ms, max_ms;  /* arrival to completion, completed requests */
    double queries_per_s;           /* completed / (last completion - first arrival) */
    double resq_per_s;              /* database residues x query residues per second */
} bp_server_metrics;

void bp_server_options_default(bp_server_options* o);
bp_status bp_server_create(bp_engine* e, const bp_db* db, const bp_server_options* opt, bp_server** out);
/* Queues a query (residue codes 1..27); any thread. */
bp_status bp_server_submit(bp_server* s, const uint8_t* query, int32_t length, uint64_t* ticket);
int32_t bp_server_state(bp_server* s, uint64_t ticket);
/* Waits for the request (timeout_ms < 0: no limit); BP_ERR_NOT_READY on timeout. */
bp_status bp_server_wait(bp_server* s, uint64_t ticket, int32_t timeout_ms);
/* The finished request's results, in the bp_result_copy layout. */
bp_status bp_server_result(bp_server* s, uint64_t ticket, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                           int64_t* n_hsps, double* latency_ms);
/* The finished request's result digest (as bp_result_digest). */
bp_status bp_server_digest(bp_server* s, uint64_t ticket, uint64_t out[2]);
/* Gives the request's device memory back to the budget. */
bp_status bp_server_release(bp_server* s, uint64_t ticket);
bp_status bp_server_stats(bp_server* s, bp_server_metrics* out);
void bp_server_destroy(bp_server* s);

/* The plain search for callers that cannot allocate device memory: a process
 * that hands out a fixed device-memory budget at start-up, a latency-critical
 * path where cudaMalloc/cudaFree would synchronise the device, or code whose
 * buffers come from an outside allocator.  No counterpart in the reference.
 *
 * The caller passes device buffers for everything: the query (d_query,
 * residues 1..27), the database (d_residues, exactly n_residues bytes: no
 * padding is read past them; d_offsets with n_subjects+1 entries running
 * from 0 to n_residues, non-decreasing, each subject below 2^29 residues --
 * checked on the device before anything is scanned), and the outputs
 * d_counters (3*n_subjects int32), d_hsp_off (n_subjects+1 int64) and d_hsps
 * (hsp_cap records).  Subjects of twice the mean length are scanned first, as
 * bp_search does.  Scratch -- neighbour table, unordered HSP records, ordering
 * cursors -- is one static 16 MiB device array in the library; the call makes
 * no cudaMalloc or cudaFree.  Limits: n_subjects <= 1,048,576, qlen <= 4096,
 * neighbour-table entries <= 1,048,576, HSPs per call <= min(hsp_cap, 262,144);
 * beyond them it returns BP_ERR_TOO_LARGE (for too many HSPs *n_hsps holds the
 * true count and the counters and offsets are complete).  The call runs on
 * `stream` (NULL: the legacy default stream) and returns when the results are
 * in place.  The first call on a device sets the array up (looks up its
 * device address and copies the scoring matrix, synchronously), so make it
 * before any stream capture.  Every call reuses the same array: calls that
 * overlap on the GPU race and must be serialised by the caller.  Returns
 * BP_OK, BP_ERR_INVALID (bad arguments, residue codes or offsets),
 * BP_ERR_TOO_LARGE (a limit above), BP_ERR_NO_DEVICE or BP_ERR_CUDA. */
bp_status bp_search_noalloc(const uint8_t* d_query, int32_t qlen, const bp_params* p, const uint8_t* d_residues,
                            int64_t n_residues, const int64_t* d_offsets, int32_t n_subjects, int32_t* d_counters,
                            int64_t* d_hsp_off, bp_hsp* d_hsps, int64_t hsp_cap, int64_t* n_hsps, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BLASTP_B200_H */
