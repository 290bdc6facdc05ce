/* fls_select.h — expression selection on the B200: the exact-size wizard and the learned selector.
 *
 * Reference counterpart: the reference picks a column's expression by encoding it with every expression of its
 * pool and keeping the smallest (ExpColEncoder<PT>::encode_all + AllExpEncodedCol::GetBest,
 * src/encoder/exp_col_encoder.cpp:18-28 and :117-129; pool src/cor/exp_pool.cpp:22-101; the Wizard::Spell
 * entry point src/wizard/wizard.cpp:19-44 leaves this choice as a TODO).  Here the choice is made per
 * (column, row-group) CHUNK of vectors (64 vectors = 64 Ki rows by default) among K = 6 no-patch candidates:
 *
 *   index  0 UNCOMPRESSED (pool id 0)   1 FFOR (id 1)   2 RLE DELTA_NO_PATCH (id 6)   3 DELTA (id 11)
 *          4 DICT FFOR (id 17)          5 DICT_RLE with raw run codes (the reference's id 27 also packs them)
 *
 * fls_sel_wizard computes the exact encoded bytes of every candidate (the pages the engine's encoders emit:
 * page header, offsets, entry points and buffers; a raw dictionary page for 4 and 5) and keeps the smallest.
 * fls_sel_learned reads 32 statistics from a sample of every chunk's vectors and runs an MLP
 * 32 -> 128 -> 128 (ReLU) -> 6 (softmax); chunks whose averaged top probability stays under a threshold go to
 * the wizard.  The MLP's forward, gradient and Adam kernels are exported for training and checking.
 *
 * All device pointers; integer columns of 32 or 64 bits (signed or not), whole 1024-value vectors, 16-byte
 * aligned.  Calls are asynchronous on the stream unless stated.  Return values are fls_status_code.
 */
#ifndef FLS_SELECT_H
#define FLS_SELECT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FLS_SEL_K 6
#define FLS_SEL_FEATURES 32
#define FLS_SEL_HIDDEN 128

typedef struct fls_sel_column {
	const void* d_values; /* n_vec * 1024 values, 16-byte aligned */
	uint64_t    n_vec;
	uint8_t     width; /* 32 or 64 */
	uint8_t     is_signed;
	uint8_t     pad[6];
} fls_sel_column;

typedef struct fls_sel_plan fls_sel_plan;

/* Chunks: every column splits into chunks of chunk_vectors vectors (the last one may be shorter), numbered
 * column by column.  Synchronous (uploads the descriptors). */
int fls_sel_plan_create(const fls_sel_column* cols, uint32_t n_cols, uint32_t chunk_vectors, fls_sel_plan** out);
int fls_sel_plan_info(const fls_sel_plan* plan, uint64_t* n_chunks, uint64_t* n_vectors);
/* host arrays of n_chunks entries: column, first vector, vector count of every chunk */
int fls_sel_plan_chunks(const fls_sel_plan* plan, uint32_t* h_col, uint64_t* h_first, uint32_t* h_count);
int fls_sel_plan_destroy(fls_sel_plan* plan);

/* String columns (no counterpart in the reference's selection code, which picks per column by trial encoding:
 * src/encoder/exp_col_encoder.cpp:18-28 over the string pool, src/cor/exp_pool.cpp:66-101).  Rows: Arrow
 * offsets (n_rows + 1, u64, device) into d_bytes (device); n_rows whole vectors.  table: HOST bytes of the
 * column's FSST symbol table in fsst_export's format, the one its DICT and FSST pages use.  A plan over string
 * columns chooses among FLS_SEL_STR_K candidates (the string pool's no-patch expressions):
 *
 *   index  0 BYTE_ARR (pool id 0)   1 DICT FFOR over an FSST dictionary (id 3)   2 FSST (id 13)
 *          3 DICT_RLE, raw run codes and a raw u16 run index (id 15)
 *
 * The wizard's sizes are exact for those pages, the dictionary holding a chunk's distinct rows in
 * first-occurrence order compressed with the column's table (distinct rows are told apart by a 64-bit hash of
 * their bytes); sizes 4 and 5 of a string chunk are UINT64_MAX.  fls_sel_wizard, fls_sel_features and
 * fls_sel_learned take the plan as they take an integer one (their statistics take the compressed length of
 * every 4th row of a sampled vector, scaled); the learned vote chooses among the 4.
 * Synchronous. */
#define FLS_SEL_STR_K 4
typedef struct fls_sel_str_column {
	const uint8_t*  d_bytes;
	const uint64_t* d_offsets;
	uint64_t        n_rows;
	const uint8_t*  table;
	uint64_t        table_size;
} fls_sel_str_column;
int fls_sel_plan_create_strings(const fls_sel_str_column* cols, uint32_t n_cols, uint32_t chunk_vectors,
                                fls_sel_plan** out);

/* Per vector (plan order: columns in order, vectors in order): bwF | bwD << 7 | bwI << 14 | runs << 19, where
 * bwF / bwD are the FFOR bit widths of the values / of their DELTA deltas, runs the runs in original order and
 * bwI the FFOR bit width of the RLE run index deltas. */
int fls_sel_vector_parts(const fls_sel_plan* plan, uint32_t* d_parts, void* stream);

/* Exact sizes (n_chunks x FLS_SEL_K, bytes) and the smallest candidate of every chunk.  d_dict_n (optional):
 * distinct values per chunk. */
int fls_sel_wizard(fls_sel_plan* plan, uint64_t* d_sizes, uint8_t* d_best, uint32_t* d_dict_n, void* stream);

/* Statistics of the sampled vectors (vectors 0, stride, 2 * stride, ... of every chunk): *n_rows rows of
 * FLS_SEL_FEATURES floats; d_row_chunk (optional) receives every row's chunk.  Pass d_feat = NULL to query
 * *n_rows.  stride 1 = every vector. */
int fls_sel_features(fls_sel_plan* plan, uint32_t stride, float* d_feat, uint32_t* d_row_chunk, uint64_t* n_rows,
                     void* stream);

/* Learned selection: statistics of the sampled vectors, MLP, per-chunk vote (mean log-probability), then the
 * wizard for chunks whose mean top probability is below threshold (threshold 0 = never).  d_choice: candidate
 * index per chunk; d_conf (optional): the mean top probability; *n_fallback (optional): chunks sent to the
 * wizard.  Synchronous. */
int fls_sel_learned(fls_sel_plan* plan, const float* d_params, uint32_t stride, float threshold, uint8_t* d_choice,
                    float* d_conf, uint64_t* n_fallback, void* stream);

/* ---- the MLP: parameters flat, W1[32][128] b1[128] W2[128][128] b2[128] W3[128][6] b3[6] ---- */
uint64_t fls_sel_param_count(void);
/* He-normal weights, zero biases (host mt19937_64 stream of the seed), uploaded to d_params.  Synchronous. */
int fls_sel_mlp_init(float* d_params, uint64_t seed);
/* class probabilities of n feature rows */
int fls_sel_mlp_forward(const float* d_params, const float* d_x, uint64_t n, float* d_prob, void* stream);
/* mean cross-entropy of n labelled rows (labels 0..5) into *d_loss and its gradient into d_grad */
int fls_sel_mlp_grad(const float* d_params, const float* d_x, const int32_t* d_y, uint64_t n, float* d_grad,
                     float* d_loss, void* stream);
/* one Adam step (step counts from 1) */
int fls_sel_adam_step(float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, float beta1, float beta2,
                      float eps, uint32_t step, void* stream);
/* Minibatch training: steps minibatches of `batch` rows, step s taking rows d_perm[s * batch ..), each step one
 * CUDA graph replay (gather, forward, backward, Adam).  d_loss_hist (optional): mean loss of every step.
 * Synchronous. */
int fls_sel_train(float* d_params, const float* d_x, const int32_t* d_y, const uint32_t* d_perm, uint32_t batch,
                  uint32_t steps, float lr, float* d_loss_hist, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLS_SELECT_H */
