/*
 * rtnn_learn.h -- learned search widths for the density-bucket partition.
 *
 * The reference picks each partition's launch radius with an analytic rule: grow a box
 * of cells until it holds K+1 points (calcSearchSize, src/optixNSearch/grid.cu:84-211)
 * and take the equal-volume sphere radius of that box (radiusFromMegacell,
 * sort.cpp:262-269; autoBatchingKNN, sort.cpp:271-320). Here a small MLP (6 -> 16 -> 16
 * -> 1, ReLU) predicts a bucket's search width from its occupancy histogram (log1p of the
 * points in cell shells 0, 1, 2, and log(K+1) - log1p(N2)), log(cell / r) and its extent.
 * Two kinds of bucket, chosen by rtnn_tuning.width_model:
 *   0  per query: the shells around the query's cell and the query's distance from the
 *      cell centre; the model predicts log(K-th distance / cell) before the query sort and
 *      the queries are bucketed by that width (one more pass, tight search boxes);
 *   1  per tile: the search's tile of 32 consecutive (Hilbert-ordered) queries, shells
 *      around the cell of the tile box's centre and the box's longest side; the model
 *      predicts log(largest K-th distance of the tile's queries / cell) and the search
 *      kernel evaluates it once per tile (no extra pass, one box per tile).
 * The width is margin * cell * exp(pred), at most r. Results never depend on the model: a
 * query that finds fewer than K neighbors inside its width is searched again wider,
 * finally at the full radius.
 *
 * The network is trained on the GPU by hand-written kernels (forward, backward, Adam)
 * on exact K-th distances produced by the plain search. All pointers are device
 * pointers. Parameters: rtnn_model_size() floats laid out as
 *   in_mean[6] in_std[6] out_mean out_std | W1[16][6] b1[16] W2[16][16] b2[16] W3[16] b3
 * (gradients cover the part after '|': rtnn_model_size() - 14 floats).
 */
#ifndef RTNN_LEARN_H_
#define RTNN_LEARN_H_

#include "rtnn.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RTNN_MODEL_FEATURES 6
#define RTNN_MODEL_HIDDEN 16
#define RTNN_MODEL_NORM_PARAMS 14

uint32_t rtnn_model_size(void);

/* Loads / reads the width model of the context (host arrays of rtnn_model_size()). */
rtnn_status rtnn_model_set(rtnn_ctx* ctx, const float* params, uint32_t n);
rtnn_status rtnn_model_get(rtnn_ctx* ctx, float* params, uint32_t n);

/* Runs the plain search (sorted rows) on one cloud and writes training samples for the
 * kind of model the context's tuning selects (width_model): per query (0), the query's six
 * features (d_feats[q][6]) and log(K-th distance / cell) (d_target[q]), a query with fewer
 * than K neighbors within r getting log(1.5 r / cell); or per tile of that search (1), the
 * tile's features (d_feats[t][6]) and log(largest K-th distance of its queries / cell)
 * (d_target[t]), queries with fewer than K neighbors within r not counting and a tile of
 * only such queries getting log(1.5 r / cell). *n_samples receives the sample count:
 * n_queries, or ceil(n_queries / 32) tiles; buffers sized for n_queries samples suffice. */
rtnn_status rtnn_collect_training(rtnn_ctx* ctx, const float* d_points, uint64_t n_points,
                                  const float* d_queries, uint64_t n_queries, rtnn_mode mode,
                                  float radius, uint32_t k, float* d_feats, float* d_target,
                                  uint64_t* n_samples);

/* Trains the context's model from scratch with Adam (mean squared error on the
 * normalised target), `batch` samples per step, in the given sample order.
 * loss_per_epoch (host, optional): mean 0.5*err^2 of each epoch. */
rtnn_status rtnn_model_train(rtnn_ctx* ctx, const float* d_feats, const float* d_target,
                             uint64_t n, uint32_t epochs, uint32_t batch, float lr,
                             uint64_t seed, float* loss_per_epoch);

/* The first-pass search width of every query under the partition (analytic, per query;
 * or, with RTNN_FLAG_LEARNED, the loaded model's width of the query's tile), in query
 * order; d_widths[q] >= radius means the full radius. Runs the whole partitioned search
 * of one cloud (rows discarded). */
rtnn_status rtnn_query_widths(rtnn_ctx* ctx, const float* d_points, uint64_t n_points,
                              const float* d_queries, uint64_t n_queries, rtnn_mode mode,
                              float radius, uint32_t k, uint32_t flags, float* d_widths);

/* Building blocks, exposed for gradient checks. d_grad receives the SUM over the batch
 * of d(0.5 * (o - t_n)^2)/d(theta) for the trained parameters; d_loss the summed loss.
 * o is the normalised network output, t_n = (target - out_mean) / out_std. */
rtnn_status rtnn_mlp_loss_grad(rtnn_ctx* ctx, const float* d_params, const float* d_feats,
                               const float* d_target, uint32_t n, float* d_grad, float* d_loss);
/* d_y[i] = out_mean + out_std * o(feats[i]) */
rtnn_status rtnn_mlp_forward(rtnn_ctx* ctx, const float* d_params, const float* d_feats,
                             uint32_t n, float* d_y);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the trained parameters with
 * gradient d_grad * grad_scale; step counts from 1. */
rtnn_status rtnn_mlp_adam_step(rtnn_ctx* ctx, float* d_params, const float* d_grad, float* d_m,
                               float* d_v, float lr, uint32_t step, float grad_scale);

#ifdef __cplusplus
}
#endif

#endif /* RTNN_LEARN_H_ */
