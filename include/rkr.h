/*
 * rkr.h -- C ABI of the B200 reverse k-ranks engine (librkr_b200.so).
 *
 * The engine answers reverse k-ranks queries over user and item embeddings with the index
 * structures of DBGroup-SUSTech/reverse-k-ranks (QSRP): per-user sampled score thresholds
 * ("SampleSearch"), per-user regression rank-bound models ("NormalLinearRegressionLP") and the SVD
 * transform ("SVD").  Results are the reference's results, bit for bit: the same users in the same
 * order with the same ranks and query scores as the reference's CPU path on the same inputs.
 *
 * Conventions.  Every function returns RKR_OK (0) or a negative status; rkr_last_error() describes
 * the last failure of the calling thread.  Nothing calls exit().  Host pointers are plain C arrays,
 * row-major; device pointers are marked d_.  One rkr_index owns one CUDA stream on one device;
 * different handles may be used from different threads, one handle from one thread at a time.
 * Reference citations are paths inside the reference project.
 */
#ifndef RKR_H
#define RKR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RKR_OK 0
#define RKR_ERR_INVALID (-1)   /* bad argument or size */
#define RKR_ERR_CUDA (-2)      /* CUDA runtime error */
#define RKR_ERR_NOMEM (-3)     /* device or host allocation failed */
#define RKR_ERR_STATE (-4)     /* the index lacks a structure the call needs */
#define RKR_ERR_IO (-5)        /* file read/write failed */

/* Query methods (the reference's --method_name values, src/app/ReverseRankIndex.cpp:107-172). */
#define RKR_METHOD_QS 0              /* src/impl/QS.hpp */
#define RKR_METHOD_QSRP_NORMAL_LP 1  /* src/impl/QSRPNormalLP.hpp */
#define RKR_METHOD_US 2              /* src/impl/US.hpp */

/* One result entry: the reference's UserRankElement (src/include/struct/UserRankElement.hpp:12-17). */
typedef struct {
    int32_t user_id;
    int32_t rank;
    float query_ip;
} rkr_user_rank;

/* Per-query counters: the reference's SingleQueryPerformance fields (src/include/util/FileIO.hpp:255-277:
 * n_prune_user, n_result_user, n_refine_user, ip_cost), the number of refinement candidates and
 * the number of items refinement examined (the reference's n_compute_item). */
typedef struct {
    int32_t n_prune;
    int32_t n_result;
    int32_t n_refine;
    int32_t n_candidate;
    int64_t n_compute_item;
    int64_t ip_cost;
} rkr_query_stats;

typedef struct rkr_index rkr_index;

const char *rkr_last_error(void);
int rkr_version(void);

/* ---- index lifecycle -------------------------------------------------------------------------- */

/* Replaces the in-memory parts of QS::BuildIndex / QSRPNormalLP::BuildIndex / US::BuildIndex
 * (src/impl/QS.hpp:259-288, src/impl/QSRPNormalLP.hpp:289-323, src/impl/US.hpp:226-242): uploads
 * the users (already L2-normalised, as readData leaves them, src/include/util/VectorIO.hpp:39-68)
 * and the data items to `device`, and prepares the norm-ordered item copy that refinement scans
 * (RefineCPUIPBound ctor, src/include/alg/DiskIndex/RefineByComputation/RefineCPUIPBound.hpp:417-467). */
int rkr_index_create(int32_t device, const float *user, int64_t n_user, const float *item, int64_t n_item,
                     int32_t dim, rkr_index **out);
int rkr_index_destroy(rkr_index *index);

/* The split dimension of the refinement bound (SVD::check_dim_, src/include/alg/SVD.hpp:126-128),
 * used by QS as well as QSRPNormalLP (src/impl/QS.hpp:267-282). */
int rkr_index_set_check_dim(rkr_index *index, int32_t check_dim);

/* SampleSearch::LoadIndex payload (src/include/alg/RankBoundRefinement/SampleSearch.hpp:199-244):
 * ranks [n_sample], ascending; thresholds [n_user][n_sample], each row descending. */
int rkr_index_load_sample_search(rkr_index *index, const int32_t *sample_rank, int32_t n_sample,
                                 const float *thresholds);

/* NormalLinearRegressionLP::LoadIndex payload (src/include/alg/RegressionPruning/
 * NormalLinearRegressionLP.hpp:448-487), one record per user: a, b, mu, sigma, error, score_max,
 * score_min (records [n_user][7]). */
int rkr_index_load_regression(rkr_index *index, const int32_t *sample_rank, int32_t n_sample,
                              const float *records);

/* SVD::LoadIndex payload (src/include/alg/SVD.hpp:258-292): transfer_item [dim][dim] and the
 * transformed users [n_user][dim]; also sets check_dim. */
int rkr_index_load_svd(rkr_index *index, int32_t check_dim, const float *transfer_item, const float *svd_user);

/* The index's SVD index as SVD::SaveIndex would write it (src/include/alg/SVD.hpp:126-188): transfer_item
 * (host [dim][dim]), the SVD-space users (host [n_user][dim]) and check_dim; any may be NULL. */
int rkr_index_svd_read(const rkr_index *index, float *transfer_item_out, float *svd_user_out, int32_t *check_dim_out);

/* Zeroes the per-user query-score vector that QSRPNormalLP carries from one query to the next
 * (Index::queryIP_l_, src/impl/QSRPNormalLP.hpp:73,109); a fresh index starts zeroed. */
int rkr_index_reset_state(rkr_index *index);

/* The regression models' level-boundary tables, built on the device when the models are loaded:
 * per user and side (0: the lower rank bound as a function of qlb, 1: the upper bound of qub) 16
 * entries (T_g, band_g), T_g the smallest binary32 score whose ComputeRankBound level
 * (NormalLinearRegressionLP.hpp:326-398; 0 -> rank 0, j + 1 -> rank[j], S + 1 -> n_item) is <= L_g,
 * band_g the half-width around T_g outside which the reference's binary32 arithmetic is guaranteed
 * to agree with the table.  levels_out: host [16], the levels L_g (0, then 14 steps to S, then
 * S + 1); tables_out: host [n_user][2][16][2] floats.  A diagnostic view of what the query kernels
 * use (no counterpart in the reference). */
int rkr_index_level_tables(rkr_index *index, int32_t *levels_out, float *tables_out);

/* Device bytes held by the index (BaseIndex::IndexSizeByte counterpart, src/include/struct/MethodBase.hpp:23). */
int rkr_index_size_bytes(const rkr_index *index, uint64_t *bytes);

/* The index's user and item counts and dimension (any may be NULL). */
int rkr_index_shape(const rkr_index *index, int64_t *n_user, int64_t *n_item, int32_t *dim);

/* Builds the thresholds for `sample_rank` on the device from the resident users and items and
 * keeps them as the index's SampleSearch table (what bsibc computes,
 * src/app/build-index/BuildSampleIndexByComputation.cpp:66-154).  thresholds_out (host,
 * [n_user][n_sample]) may be NULL. */
int rkr_index_build_sample_search(rkr_index *index, const int32_t *sample_rank, int32_t n_sample,
                                  float *thresholds_out);

/* ---- query -------------------------------------------------------------------------------------- */

/* BaseIndex::Retrieval (src/include/struct/MethodBase.hpp:16-18) for `method` over host query
 * vectors [n_query][dim].  out: host [n_answered][topk]; stats: host [n_answered] or NULL.
 * US answers only the first 100 queries when n_sample <= 1000, as the reference does
 * (src/impl/US.hpp:113); *n_answered says how many rows were written.  topk > n_user is
 * RKR_ERR_INVALID (the reference exits, src/impl/QS.hpp:116-119); so is topk > 4096, the largest
 * top-k the device assembly holds. */
int rkr_retrieval(rkr_index *index, int32_t method, const float *query, int32_t n_query, int32_t topk,
                  rkr_user_rank *out, rkr_query_stats *stats, int32_t *n_answered);

/* Same, with the queries and outputs already in device memory of the index's device; runs on
 * `stream` (a cudaStream_t, or NULL for the index's own stream) and returns after the work is
 * enqueued and the result is complete on that stream. */
int rkr_retrieval_device(rkr_index *index, int32_t method, const float *d_query, int32_t n_query, int32_t topk,
                         rkr_user_rank *d_out, rkr_query_stats *d_stats, int32_t *n_answered, void *stream);

/* BaseIndex::Retrieval with a top-k per query, the serving boundary's form (the reference answers
 * one topk per Retrieval call, src/app/ReverseRankIndex.cpp:191-192, src/impl/QSRPNormalLP.hpp:116-118;
 * a batch here may mix them): query i of the answered ones gets k_per_q[i] entries, written after
 * those of queries 0 .. i-1 (out holds sum(k_per_q[0 .. n_answered)) entries).  The results equal
 * those of one rkr_retrieval call per query in order with topk = k_per_q[i] (the carried
 * QSRPNormalLP scores advance the same way).  Every k must be in [1, min(n_user, 4096)]. */
int rkr_query(rkr_index *index, int32_t method, const float *query, int32_t n_query, const int32_t *k_per_q,
              rkr_user_rank *out, rkr_query_stats *stats, int32_t *n_answered);

/* Same, with the queries and outputs in device memory (k_per_q stays a host array); runs on `stream`
 * (or the index's own when NULL) and returns once the result is complete on that stream. */
int rkr_query_device(rkr_index *index, int32_t method, const float *d_query, int32_t n_query,
                     const int32_t *k_per_q, rkr_user_rank *d_out, rkr_query_stats *d_stats, int32_t *n_answered,
                     void *stream);

/* ---- serving ------------------------------------------------------------------------------------- */

/* A persistent serving loop over a resident index (no counterpart in the reference, whose query app
 * answers one query file per run, src/app/ReverseRankIndex.cpp:83-220).  Requests -- each a set of
 * query items with a top-k per item -- queue in arrival order; n_workers workers, each on its own
 * CUDA stream and work arrays over the shared resident index, take requests from the head of the
 * queue while they fit a batch (at most max_batch_queries items, and at most as many as the
 * workspace_bytes memory budget holds at about 2 bytes per (query item, user) pair; 0: no memory
 * limit beyond the slots), pad the batch to the next power of two from 16 to 4096 and replay
 * the CUDA graph captured for that size.  Each request gets the result a fresh index would give it
 * alone (QSRPNormalLP's carried per-user scores, QSRPNormalLP.hpp:73,109,213-218, are scoped to the
 * request), whatever it is batched with.  Methods: QS and QSRPNormalLP.  The index must stay loaded
 * and unchanged while a server uses it; the server only reads it. */
typedef struct {
    int32_t method;             /* RKR_METHOD_QS or RKR_METHOD_QSRP_NORMAL_LP */
    int32_t max_batch_queries;  /* query items per batch, 1 .. 4096 */
    int32_t n_workers;          /* batches in flight, 1 .. 8 */
    int32_t reserved;
    int64_t workspace_bytes;    /* per-worker memory budget for a batch's work arrays (0: none) */
} rkr_server_config;
typedef struct rkr_server rkr_server;

int rkr_server_create(rkr_index *index, const rkr_server_config *config, rkr_server **out);
/* Queues a request (copies the query items [n_query][dim] and k_per_q); *ticket names it.  n_query
 * must fit one batch. */
int rkr_server_submit(rkr_server *server, const float *query, int32_t n_query, const int32_t *k_per_q,
                      uint64_t *ticket);
/* Waits (timeout_s < 0: without limit) for a request and copies its results: out holds sum(k_per_q)
 * entries laid out as rkr_query's, stats n_query entries (either may be NULL); latency_s, if not
 * NULL, receives {submit to done, submit to start} in seconds.  A ticket is waited for once. */
int rkr_server_wait(rkr_server *server, uint64_t ticket, double timeout_s, rkr_user_rank *out,
                    rkr_query_stats *stats, double *latency_s);
/* Batches run, requests and query items answered, padding items added, and the workers' summed busy
 * time since the server started. */
int rkr_server_counters(rkr_server *server, int64_t *batches, int64_t *requests, int64_t *queries,
                        int64_t *padded, double *busy_s);
/* Answers every queued request, then stops the workers and frees their resources. */
int rkr_server_destroy(rkr_server *server);

/* ---- measurement ---------------------------------------------------------------------------------- */

/* Per-kernel device time: with profiling on, every kernel the index launches is bracketed by CUDA
 * events on the stream it runs on.  rkr_profile_read returns, per kernel name, the summed time and
 * the launch count since the previous complete read (a read with max_kernels >= *n_kernels clears
 * them; a smaller one only reports the count); names is [max_kernels][64] chars.  Entries whose
 * name ends in "_pairs", "_queries" or "_rows" are counters rather than kernels (time 0, `launches` holds
 * the count): two_pass_compaction_queries counts the queries whose flagged users outgrew the sparse
 * compaction's list and took the two-pass form (two_pass_need_to_2x_queries, _to_4x_, _to_16x_ and
_beyond_ count them by how far their flagged users exceed the list);
 * screen_undecided_pairs counts the (query, user) pairs whose regression levels or threshold group
 * the screens (tensor-core scores with an error bound, the fast binary32 CDF) left to the
 * reference's own arithmetic; rescored_pairs the pairs whose score a later pass recomputed (a fine
 * threshold bucket within the bound, a reported or carried score); refine_exact_pairs the
 * refinement's (candidate, item) tests the tensor-core bound left undecided; row_select_deferred_rows
 * the build's score rows that the streaming selection of long rows left to the scatter form.
 * (The reference's counterpart is its TimeRecord per stage, src/include/util/TimeMemory.hpp:7-24.) */
int rkr_profile_enable(rkr_index *index, int32_t on);
int rkr_profile_read(rkr_index *index, int32_t max_kernels, char *names, double *total_ms, int64_t *launches,
                     int32_t *n_kernels);

/* Diagnostics of the tensor-core pair scores: for n_query (<= 4096) host queries, out (host,
 * [n_query][n_user][2] floats) receives each (query, user) pair's estimate of its full score (SVD
 * space for QSRPNormalLP, as the reference scores round 2) and the bound the kernel holds on its
 * distance to the reference's binary32 score; NaN where the estimate path did not run (shapes the
 * exact tiles take).  Runs one pass of the query pipeline on the index's stream (its results are
 * discarded; the carried QSRPNormalLP scores are restored).  No counterpart in the reference. */
int rkr_score_estimates(rkr_index *index, int32_t method, const float *query, int32_t n_query, float *out);

/* ---- index build --------------------------------------------------------------------------------- */

/* ComputeScoreTableBatch::ComputeSortItemsBatch (src/include/score_computation/ComputeScoreTableBatch.hpp:79-92):
 * rows_out (host, [n_rows][n_item]) = scores of users [start, start + n_rows) against all items,
 * each row sorted descending. */
int rkr_score_sort_batch(rkr_index *index, int64_t start_user, int64_t n_rows, float *rows_out);

/* ComputeQueryRankByComputation (src/app/build-index/QueryRankByComputation.hpp:122-242):
 * accu_out (host, [n_sample_item][n_item + 1]) is, for each sampled item, the cumulative count of
 * users by the item's rank (number of items scoring strictly above it). */
int rkr_index_query_rank_distribution(rkr_index *index, const int32_t *sample_item, int32_t n_sample_item,
                                      int32_t *accu_out);

/* Threshold build that allocates nothing.  Some callers cannot let a library call cudaMalloc:
 * services that fix their device footprint at start-up, code running under a caching allocator
 * or a carved-up memory pool, callers inside allocation-sensitive sections.  This entry point
 * computes the same thresholds as rkr_index_build_sample_search, for users and items already in
 * device memory of the current device (d_user [n_user][dim], d_item [n_item][dim], d_thresholds
 * [n_user][n_sample] written), with host sample ranks (ascending, in [0, n_item)).  Its only
 * scratch is a fixed 32 MiB array compiled into the library, which every GPU that loads the
 * library keeps until the process exits; it holds at most 16384 sample ranks and batches of
 * (32 MiB - 64 KiB) / (4 * round_up(n_item, 4)) score rows, and n_item must also fit the
 * shared-memory row selection (about 24,000 items on B200); larger sizes are RKR_ERR_INVALID.
 * Every call looks up the array's device address in the current device's context
 * (cudaGetSymbolAddress), so the address stays right after a device reset.  Calls share the
 * array: calls that overlap on
 * the GPU (other streams, other host threads) race; the call returns after its work on `stream`
 * (a cudaStream_t, NULL for the legacy default stream) has finished.  There is no counterpart in
 * the reference, which always allocates its score-table buffers. */
int rkr_build_thresholds_static(const float *d_user, int64_t n_user, const float *d_item, int64_t n_item,
                                int32_t dim, const int32_t *sample_rank, int32_t n_sample, float *d_thresholds,
                                void *stream);

/* Host-side build steps (CPU; no device needed). */

/* VectorMatrix::vectorNormalize (src/include/struct/VectorMatrix.hpp:51-66), in place. */
int rkr_normalize(float *vectors, int64_t n, int32_t dim);
/* SampleItem (src/app/build-index/QueryRankBySample.hpp:20-37): mt19937(0) shuffle of item ids. */
int rkr_sample_item(int32_t n_item, int32_t n_sample_item, int32_t *out);
/* ComputeSortKthRank (src/app/build-index/QueryRankBySample.hpp:103-134). */
int rkr_sort_kth_rank(const int32_t *accu, int64_t n_item, int32_t n_sample_item, int32_t sample_topk,
                      int32_t *sort_kth_out, int32_t *sort_sample_id_out);
/* FindOptimalSampleFast with the OptimalPart candidates
 * (src/include/alg/RankBoundRefinement/FindSampleRank/OptimalSampleRankFast.hpp:269-472);
 * sort_kth ascending, accu_sorted rows in that order. */
int rkr_find_optimal_sample_rank(int64_t n_user, int64_t n_item, int32_t n_sample, int32_t n_sample_query,
                                 const int32_t *sort_kth, const int32_t *accu_sorted, int32_t *out,
                                 int64_t *train_cost);
/* FindUniformSample (src/include/alg/RankBoundRefinement/FindSampleRank/UniformSample.hpp:17-56). */
int rkr_uniform_sample_rank(int32_t n_item, int32_t n_sample, int32_t *out);
/* NormalLinearRegressionLP fit (StartPreprocess / BatchLoopPreprocess,
 * NormalLinearRegressionLP.hpp:72-310): records_out [n_user][7] as rkr_index_load_regression takes. */
int rkr_fit_regression(const float *thresholds, int64_t n_user, int32_t n_sample, float *records_out);
/* The same fit on the device, from the index's resident sampled thresholds (loaded or built), with
 * the index's sample ranks as the models' (NormalLinearRegressionLP::BuildIndex fits from the
 * SampleSearch index of the same ranks): the models become the index's regression index (as
 * rkr_index_load_regression would load them) and, if records_out (host, [n_user][7]) is not NULL,
 * are copied out.  The records equal rkr_fit_regression's (the same arithmetic, operation by
 * operation).  2 <= n_sample <= 4096. */
int rkr_index_fit_regression(rkr_index *index, float *records_out);
/* SVD::PerformSVD (src/include/alg/SVD.hpp:62-124): thin SVD of the users, the transfer matrix,
 * the transformed users and check_dim for the given sigma ratio. */
int rkr_svd_build(const float *user, int64_t n_user, int32_t dim, float sigma, float *transfer_item_out,
                  float *svd_user_out, int32_t *check_dim_out);
/* The same transform built on the device from the index's resident users (the Gram matrix and the
 * projection on the device, the d x d eigen-decomposition on the host) and made the index's SVD
 * index, as rkr_index_load_svd would load it; transfer_item_out (host [dim][dim]), svd_user_out
 * (host [n_user][dim]) and check_dim_out may be NULL.  A valid transform like rkr_svd_build's (the
 * Gram matrix's sums run in another order, so the two agree to rounding, not bit for bit); the same
 * users give the same transform on every run (the Gram matrix's partial sums are added in a fixed
 * order).  A user shard is RKR_ERR_STATE: its transform must be every shard's. */
int rkr_index_svd_build(rkr_index *index, float sigma, float *transfer_item_out, float *svd_user_out,
                        int32_t *check_dim_out);

/* ---- index files --------------------------------------------------------------------------------- */

/* The reference's on-disk index layouts, read and written byte for byte (native-endian size_t, int
 * and float, no padding).  A missing, short or inconsistent file is RKR_ERR_IO; nothing here touches
 * the GPU.  Each *_info call reads only the header, so that the caller can size the buffers of the
 * matching read; output buffers may be NULL to skip a part. */

/* SampleSearch::SaveIndex / LoadIndex (src/include/alg/RankBoundRefinement/SampleSearch.hpp:158-244):
 * size_t n_sample, n_item, n_user; int rank[n_sample]; float thresholds[n_user][n_sample] (the
 * memory_index form; the qrs_to_sample_index form that fsr writes ends after the ranks:
 * *has_scores = 0, and writing with thresholds = NULL produces it). */
int rkr_file_sample_search_info(const char *path, int32_t *n_sample, int64_t *n_item, int64_t *n_user,
                                int32_t *has_scores);
int rkr_file_read_sample_search(const char *path, int32_t *rank_out, float *thresholds_out);
int rkr_file_write_sample_search(const char *path, const int32_t *rank, int32_t n_sample, int64_t n_item,
                                 int64_t n_user, const float *thresholds);

/* NormalLinearRegressionLP::SaveIndex / LoadIndex (src/include/alg/RegressionPruning/
 * NormalLinearRegressionLP.hpp:419-487): size_t n_item, n_user; int n_sample; int rank[n_sample];
 * float (a, b)[n_user], (mu, sigma)[n_user], err[n_user], (smax, smin)[n_user].  Records here are
 * [n_user][7] = a, b, mu, sigma, err, smax, smin, as rkr_index_load_regression takes them. */
int rkr_file_regression_info(const char *path, int32_t *n_sample, int64_t *n_item, int64_t *n_user);
int rkr_file_read_regression(const char *path, int32_t *rank_out, float *records_out);
int rkr_file_write_regression(const char *path, const int32_t *rank, int32_t n_sample, int64_t n_item,
                              int64_t n_user, const float *records);

/* SVD::SaveIndex / LoadIndex (src/include/alg/SVD.hpp:126-188): size_t n_user, n_item, dim; float
 * sigma; int check_dim; float transfer_item[dim][dim], svd_user[n_user][dim], svd_item[n_item][dim]
 * (svd_item = NULL on write: zeros, a part the query path never reads). */
int rkr_file_svd_info(const char *path, int64_t *n_user, int64_t *n_item, int32_t *dim, float *sigma,
                      int32_t *check_dim);
int rkr_file_read_svd(const char *path, float *transfer_item, float *svd_user, float *svd_item);
int rkr_file_write_svd(const char *path, int64_t n_user, int64_t n_item, int32_t dim, float sigma, int32_t check_dim,
                       const float *transfer_item, const float *svd_user, const float *svd_item);

/* The query-distribution directory (WriteDistributionBelowTopk, src/app/build-index/FileIO.hpp:57-137;
 * read back as ReadQueryDistribution does, OptimalSampleRank.hpp:157-200): dir/sample_itemID_l.txt
 * (the sampled item ids in sorted-sample order, one per line), dir/sort_kth_rank_l.index
 * (int[n_sample_item]) and dir/accu_n_user_rank_l.index (the accu rows, [n_sample_item][n_item + 1]
 * ints, in sorted-sample order).  The write takes what rkr_sample_item,
 * rkr_index_query_rank_distribution and rkr_sort_kth_rank return (accu in sample order) and creates
 * dir if needed; the read returns the file order. */
int rkr_file_write_query_distribution(const char *dir, const int32_t *sample_item, const int32_t *sort_kth_rank,
                                      const int32_t *sort_sample_id, const int32_t *accu, int32_t n_sample_item,
                                      int64_t n_item);
int rkr_file_read_query_distribution(const char *dir, int32_t n_sample_item, int64_t n_item, int32_t *sample_item_out,
                                     int32_t *sort_kth_rank_out, int32_t *accu_out);

/* Loads the file set the reference's factories read (QS::BuildIndex, src/impl/QS.hpp:259-288;
 * QSRPNormalLP::BuildIndex, src/impl/QSRPNormalLP.hpp:289-323; US::BuildIndex, src/impl/US.hpp)
 * from index_dir into the index: the SampleSearch index (memory_index/QS-<dataset>-n_sample_..
 * -n_sample_query_..-sample_topk_...index, or memory_index/US-<dataset>-n_sample_...index for US),
 * for QS the check_dim of svd_index/<dataset>.index, for QSRPNormalLP that SVD index and the
 * regression index (memory_index/NormalLinearRegressionLP-QS-<dataset>-...index).  The files are
 * memory-mapped and copied to the device from the maps; their user counts must match the index's. */
int rkr_index_load_files(rkr_index *index, int32_t method, const char *index_dir, const char *dataset_name,
                         int32_t n_sample, int32_t n_sample_query, int32_t sample_topk);

/* bstb's disk score table (src/app/BuildScoreTableBatch.cpp:75-150, written by ReadAll::BuildIndexLoop,
 * src/include/alg/DiskIndex/ReadAll.hpp): path receives the first n_user_out (<= n_user) users'
 * score rows against all items, each sorted descending, n_item floats per row, no header (the
 * reference names it <index_dir>/<dataset>.index and caps the users at its evaluation size).  The
 * rows are computed on the device, as rkr_score_sort_batch returns them. */
int rkr_file_write_score_table(rkr_index *index, const char *path, int64_t n_user_out);

/* ---- updates ---------------------------------------------------------------------------------------- */

/* QSRPNormalLPUpdate::InsertUser (src/impl/Update/QSRPNormalLPUpdate.hpp:308-347): appends n users
 * (host [n][dim], L2-normalised) as users n_user .. n_user + n - 1, with their sampled thresholds
 * (the index's sample ranks) and, when the index has regression models, their models, computed on
 * the device; an index with an SVD transform gets it rebuilt over every user with sigma, and its
 * check_dim with it (SVDUpdate::InsertUser, src/include/alg/SVDUpdate.hpp:63-79).  The new users'
 * carried QSRPNormalLP scores are zero.  The index must have sampled thresholds, and its regression
 * models (if any) the thresholds' sample ranks.  No other call may use the index meanwhile. */
int rkr_index_insert_users(rkr_index *index, const float *user, int64_t n, float sigma);

/* QSRPNormalLPUpdate::DeleteUser (:349-365): removes the users ids[0 .. n) (any order, no repeats,
 * fewer than n_user); the others keep their order (ids close up), thresholds, models and SVD-space
 * rows, and the transform stays (SVDUpdate.hpp:81-84).  The carried QSRPNormalLP scores are resized
 * as the reference resizes its vector: the first n_user - n entries stay, whichever users they
 * belonged to.  No other call may use the index meanwhile.  Item insertion and deletion
 * (SampleSearchUpdate's rank offsets) are not supported. */
int rkr_index_delete_users(rkr_index *index, const int64_t *ids, int64_t n);

/* ---- user shards ---------------------------------------------------------------------------------- */
/*
 * An index too large for one GPU is split by users: shard s is an ordinary rkr_index over the
 * contiguous users [user_offset_s, user_offset_s + n_user_s) of n_user_total (ascending offsets by
 * shard number), with the same items, sample ranks and SVD transform, and with its users' rows of the
 * thresholds, regression records and SVD-space users.  The reference's one global step,
 * PruneCandidateByBound (src/include/alg/RankBoundRefinement/PruneCandidateByBound.hpp:19-179), needs
 * the k-th smallest rank bound over all users; every selection of the engine reads that k-th value
 * off a small per-query count array (levels, groups, buckets), so the shards sum those arrays
 * element-wise and select alike, then classify, refine and assemble their own users.  The host
 * merges the shards' partial rows (rkr_shard_merge).  There is no counterpart in the reference,
 * which holds every user in one process.
 */

/* Element-wise sum over all shards of n int32 counts, in place.  counts is device memory of the
 * calling shard's GPU (host memory when stream is NULL and the caller is host code), ordered after
 * the work already queued on stream (a cudaStream_t); the counts must be summed before any later
 * work on that stream reads them (stream-ordered, or by waiting).  Returns 0, or non-zero to fail
 * the query.  Every shard makes the same calls in the same order with the same n. */
typedef int (*rkr_exchange_fn)(void *ctx, int32_t *counts, int64_t n, void *stream);

/* Makes index shard `shard` of n_shards (users [user_offset, user_offset + its n_user) of
 * n_user_total), summing counts through exchange(ctx, ...).  n_shards == 1 with exchange NULL
 * makes the index whole again.  A shard answers rkr_shard_query only (rkr_retrieval / rkr_query /
 * serving are RKR_ERR_STATE on it); rkr_index_query_rank_distribution returns the sum over all
 * shards (every shard must call it). */
int rkr_index_set_shard(rkr_index *index, int32_t shard, int32_t n_shards, int64_t user_offset,
                        int64_t n_user_total, rkr_exchange_fn exchange, void *ctx);

/* This shard's part of rkr_query: every shard calls it with the same queries and k_per_q (host
 * arrays).  part (host, sum(k_per_q) entries laid out as rkr_query's out) receives, per query,
 * n_front[q] of this shard's result users in user-id order, then this shard's refined candidates
 * sorted by (rank, user id), at most k entries in all; unused entries have user_id -1.  User ids
 * are global (user_offset added).  stats (host, or NULL) receives the global n_prune and n_result
 * and this shard's share of the other counters (shard 0 also counts the refinement-independent
 * part of ip_cost). */
int rkr_shard_query(rkr_index *index, int32_t method, const float *query, int32_t n_query, const int32_t *k_per_q,
                    rkr_user_rank *part, int32_t *n_front, rkr_query_stats *stats, int32_t *n_answered);

/* Merges the shards' parts (in shard order) into rkr_query's output: the result users of all
 * shards in user-id order, then the candidates of all shards by (rank, user id), k per query, as
 * the reference assembles them (src/impl/QSRPNormalLP.hpp:213-226, src/impl/QS.hpp:185-198).
 * parts[s], n_fronts[s] and stats[s] (stats may be NULL) are shard s's outputs; stats_out may be
 * NULL.  Host only. */
int rkr_shard_merge(int32_t n_shards, int32_t n_query, const int32_t *k_per_q, const rkr_user_rank *const *parts,
                    const int32_t *const *n_fronts, const rkr_query_stats *const *stats, rkr_user_rank *out,
                    rkr_query_stats *stats_out);

/* An exchange for shards driven by threads of one process (for example several shards on one
 * GPU, or one per GPU from one process): rkr_host_exchange is an rkr_exchange_fn whose ctx is a
 * group from rkr_host_exchange_create.  Each call waits for the stream, copies the counts to the
 * host, waits up to timeout_s for every member's call (or fails), sums and copies back. */
int rkr_host_exchange_create(int32_t n_members, double timeout_s, void **group);
int rkr_host_exchange(void *group, int32_t *counts, int64_t n, void *stream);
int rkr_host_exchange_destroy(void *group);

#ifdef __cplusplus
}
#endif
#endif /* RKR_H */
