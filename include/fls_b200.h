/* fls_b200.h — C ABI of the B200-native FastLanes decode engine.
 *
 * Drop-in boundary for the decode path of cwida/FastLanes.  Every entry point below names the reference
 * interface it replaces (paths are inside the reference project).  All pointers named d_* are device
 * pointers; calls with an fls_stream_t are asynchronous on that stream (NULL = legacy default stream) and
 * return a status code for argument errors detected on the host.  Errors found on the device (corrupt
 * input) are OR-ed into a per-device status word read by fls_gpu_status().
 *
 * Vector layout: 1024 values per vector in the FastLanes unified transposed layout
 *   transposed[k] = original[(k % 16) * 64 + O[(k / 16) % 8] * 8 + k / 128],  O = {0,4,2,6,1,5,3,7}.
 * order = FLS_TRANSPOSED leaves outputs in that layout (what the reference primitives return);
 * order = FLS_ORIGINAL also untransposes (what Materializer::Materialize, src/encoder/materializer.cpp:13-21,
 * returns).
 */
#ifndef FLS_B200_H
#define FLS_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* fls_stream_t; /* a cudaStream_t */

enum fls_status_code {
	FLS_OK              = 0,
	FLS_ERR_ARG         = -1, /* null pointer, bad size, bad order, misaligned buffer */
	FLS_ERR_CUDA        = -2, /* a CUDA runtime call failed */
	FLS_ERR_FORMAT      = -3, /* malformed page / dictionary bytes */
	FLS_ERR_UNSUPPORTED = -4, /* expression or type outside the decode path */
	FLS_ERR_BW          = -5, /* bit width above the type width */
	FLS_ERR_TOO_LARGE   = -6, /* input beyond the fixed scratch of an allocation-free entry point */
};

enum fls_order_code { FLS_TRANSPOSED = 0, FLS_ORIGINAL = 1 };

/* Device status bits (fls_gpu_status) */
#define FLS_DEV_TIMEOUT 1
#define FLS_DEV_BAD_BW 2
#define FLS_DEV_BAD_INDEX 4
#define FLS_DEV_BAD_LAYOUT 8

/* Synchronise the current device and return the OR of all device status bits raised since the last reset. */
int fls_gpu_status(int reset);

/* Number of kernels this library has launched since the last reset (for launch accounting in benchmarks). */
uint64_t fls_gpu_launch_count(int reset);

/* Failure injection for tests of the bounded waits (no counterpart in the reference): fls_gpu_unffor_u32 over
 * n_vec vectors (d_in 16-byte aligned) in which vector stall_vector's staging copy has its byte count armed on
 * the mbarrier but is never issued, so nothing is in flight and that wait runs out after spin_limit polls (> 0);
 * the warp then raises FLS_DEV_TIMEOUT, waits for the copies it did issue and leaves; every other vector decodes.
 * No GPU fault is involved and the context stays usable. */
int fls_gpu_test_stalled_copy(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint32_t* d_base,
                              const uint64_t* d_byte_off, uint64_t n_vec, uint64_t stall_vector, uint32_t spin_limit,
                              fls_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Primitives, batched over n_vec vectors.
 *   d_bw[v]        bit width of vector v (0..W)
 *   d_byte_off[v]  byte offset of vector v's packed words inside d_in (NULL: vector v starts at v*bw[v]*128,
 *                  which is only meaningful when every vector has the same width)
 *   d_base[v]      FOR base of vector v (unffor)
 *   d_lane_base    L = 1024/W lane bases per vector, 128 bytes per vector (rsum)
 * Packed words of a vector start at a 4-byte boundary at least; 16-byte aligned vectors are staged by TMA.
 * ------------------------------------------------------------------------------------------------------- */

/* replaces generated::unpack::fallback::scalar::unpack (include/fls_gen/unpack/unpack.hpp:6-11) */
int fls_gpu_unpack_u8(const uint8_t* d_in, uint8_t* d_out, const uint8_t* d_bw, const uint64_t* d_byte_off,
                      uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unpack_u16(const uint16_t* d_in, uint16_t* d_out, const uint8_t* d_bw, const uint64_t* d_byte_off,
                       uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unpack_u32(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint64_t* d_byte_off,
                       uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unpack_u64(const uint64_t* d_in, uint64_t* d_out, const uint8_t* d_bw, const uint64_t* d_byte_off,
                       uint64_t n_vec, int order, fls_stream_t stream);

/* replaces generated::unffor::fallback::scalar::unffor (include/fls_gen/unffor/unffor.hpp:6-18) */
int fls_gpu_unffor_u8(const uint8_t* d_in, uint8_t* d_out, const uint8_t* d_bw, const uint8_t* d_base,
                      const uint64_t* d_byte_off, uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unffor_u16(const uint16_t* d_in, uint16_t* d_out, const uint8_t* d_bw, const uint16_t* d_base,
                       const uint64_t* d_byte_off, uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unffor_u32(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint32_t* d_base,
                       const uint64_t* d_byte_off, uint64_t n_vec, int order, fls_stream_t stream);
int fls_gpu_unffor_u64(const uint64_t* d_in, uint64_t* d_out, const uint8_t* d_bw, const uint64_t* d_base,
                       const uint64_t* d_byte_off, uint64_t n_vec, int order, fls_stream_t stream);

/* replaces generated::rsum::fallback::scalar::rsum (include/fls_gen/rsum/rsum.hpp:9-12); d_in holds 1024
 * transposed deltas per vector */
int fls_gpu_rsum_u8(const uint8_t* d_in, uint8_t* d_out, const uint8_t* d_lane_base, uint64_t n_vec, int order,
                    fls_stream_t stream);
int fls_gpu_rsum_u16(const uint16_t* d_in, uint16_t* d_out, const uint16_t* d_lane_base, uint64_t n_vec,
                     int order, fls_stream_t stream);
int fls_gpu_rsum_u32(const uint32_t* d_in, uint32_t* d_out, const uint32_t* d_lane_base, uint64_t n_vec,
                     int order, fls_stream_t stream);
int fls_gpu_rsum_u64(const uint64_t* d_in, uint64_t* d_out, const uint64_t* d_lane_base, uint64_t n_vec,
                     int order, fls_stream_t stream);

/* fused unffor + rsum: the DELTA decode of ffor_decompress + rsum_decompress
 * (src/cor/prm/ffor/ffor_decompress.cpp:13-32, src/cor/prm/rsum/rsum_decompress.cpp:12-24) */
int fls_gpu_unffor_rsum_u16(const uint16_t* d_in, uint16_t* d_out, const uint8_t* d_bw, const uint16_t* d_base,
                            const uint16_t* d_lane_base, const uint64_t* d_byte_off, uint64_t n_vec, int order,
                            fls_stream_t stream);
int fls_gpu_unffor_rsum_u32(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint32_t* d_base,
                            const uint32_t* d_lane_base, const uint64_t* d_byte_off, uint64_t n_vec, int order,
                            fls_stream_t stream);
int fls_gpu_unffor_rsum_u64(const uint64_t* d_in, uint64_t* d_out, const uint8_t* d_bw, const uint64_t* d_base,
                            const uint64_t* d_lane_base, const uint64_t* d_byte_off, uint64_t n_vec, int order,
                            fls_stream_t stream);

/* replaces generated::untranspose::fallback::scalar::untranspose_i / _o
 * (include/fls_gen/untranspose/untranspose.hpp:8-19) */
int fls_gpu_untranspose_i_u8(const uint8_t* d_in, uint8_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_untranspose_i_u16(const uint16_t* d_in, uint16_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_untranspose_i_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_untranspose_i_u64(const uint64_t* d_in, uint64_t* d_out, uint64_t n_vec, fls_stream_t stream);

/* Encoder side (fixtures, trial encodes): generated::transpose::...::transpose_i
 * (include/fls_gen/transpose/transpose.hpp:8-19), generated::ffor::...::ffor (include/fls_gen/ffor/ffor.hpp:6-15),
 * generated::unrsum::...::unrsum (include/fls_gen/unrsum/unrsum.hpp:8-16) and the base/bit-width choice of
 * ffor_analyze (src/cor/prm/ffor/ffor_analyze.cpp:77-102; exact bit count, signed min/max when is_signed). */
int fls_gpu_transpose_i_u8(const uint8_t* d_in, uint8_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_transpose_i_u16(const uint16_t* d_in, uint16_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_transpose_i_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_transpose_i_u64(const uint64_t* d_in, uint64_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_ffor_u8(const uint8_t* d_in, uint8_t* d_out, const uint8_t* d_bw, const uint8_t* d_base,
                    const uint64_t* d_byte_off, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_ffor_u16(const uint16_t* d_in, uint16_t* d_out, const uint8_t* d_bw, const uint16_t* d_base,
                     const uint64_t* d_byte_off, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_ffor_u32(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint32_t* d_base,
                     const uint64_t* d_byte_off, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_ffor_u64(const uint64_t* d_in, uint64_t* d_out, const uint8_t* d_bw, const uint64_t* d_base,
                     const uint64_t* d_byte_off, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_unrsum_u16(const uint16_t* d_in, uint16_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_unrsum_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_unrsum_u64(const uint64_t* d_in, uint64_t* d_out, uint64_t n_vec, fls_stream_t stream);
int fls_gpu_analyze_u16(const uint16_t* d_in, uint8_t* d_bw, uint16_t* d_base, uint64_t n_vec, int is_signed,
                        fls_stream_t stream);
int fls_gpu_analyze_u32(const uint32_t* d_in, uint8_t* d_bw, uint32_t* d_base, uint64_t n_vec, int is_signed,
                        fls_stream_t stream);
int fls_gpu_analyze_u64(const uint64_t* d_in, uint8_t* d_bw, uint64_t* d_base, uint64_t n_vec, int is_signed,
                        fls_stream_t stream);


/* ---------------------------------------------------------------------------------------------------------
 * Batched decode plans.  A plan describes many vector batches (any mix of widths and encodings) and the
 * order in which the persistent decode kernel takes their vectors.  Creating a plan uploads its descriptors
 * and queue once; fls_plan_decode then only launches (one kernel, capturable in a CUDA graph).
 * Replaces the per-vector Engine/Exe dispatch (src/cor/eng/executor.cpp:44-53) with a device-side queue of
 * (batch, vector) work items.
 * ------------------------------------------------------------------------------------------------------- */
enum fls_encoding_code { FLS_ENC_RAW = 0, FLS_ENC_FFOR = 1, FLS_ENC_DELTA = 2 };

typedef struct {
	uint8_t         width;    /* 8, 16, 32 or 64 */
	uint8_t         encoding; /* fls_encoding_code */
	uint8_t         order;    /* fls_order_code */
	uint8_t         reserved;
	uint32_t        n_vec;
	const void*     d_packed;    /* packed words of all vectors */
	const uint64_t* d_byte_off;  /* per-vector byte offset in d_packed */
	const uint8_t*  d_bw;        /* per-vector bit width (FFOR/DELTA) */
	const void*     d_base;      /* per-vector FOR base (FFOR/DELTA) */
	const void*     d_lane_base; /* per-vector 128-byte lane bases (DELTA) */
	void*           d_out;       /* n_vec * 1024 values */
} fls_vector_batch;

typedef struct fls_plan fls_plan;

/* d_queue: n_items work items (batch << 24 | vector), NULL = every vector of every batch in batch order.
 * The queue is copied; the batches' device buffers must outlive the plan. */
int fls_plan_create(const fls_vector_batch* batches, uint32_t n_batches, const uint32_t* d_queue, uint64_t n_items,
                    fls_plan** out_plan);
/* flags of fls_plan_create_ex; fls_plan_create groups the queue by vector kind (flags = 0) */
#define FLS_PLAN_KEEP_ORDER 1u /* take the work items exactly in queue order */
int fls_plan_create_ex(const fls_vector_batch* batches, uint32_t n_batches, const uint32_t* d_queue,
                       uint64_t n_items, uint32_t flags, fls_plan** out_plan);
int fls_plan_decode(const fls_plan* plan, fls_stream_t stream);
/* Same, with an explicit grid (CTAs); 0 = one wave of resident CTAs. */
int fls_plan_decode_grid(const fls_plan* plan, int grid, fls_stream_t stream);
int fls_plan_destroy(fls_plan* plan);
/* Shape of the kernel a plan launches (its first segment): threads per CTA, dynamic shared memory, resident CTAs
 * per SM. */
int fls_plan_geometry(const fls_plan* plan, int* threads, int* smem_bytes, int* ctas_per_sm);
/* Autotuner (no reference counterpart): times every geometry variant (warps per CTA x TMA staging depth, hence
 * vectors per warp) of the plan's kernel families on the plan's own data, `reps` launches each, and keeps the
 * fastest per launch segment.  Runs decodes (the outputs are written).  Synchronous. */
int fls_plan_autotune(fls_plan* plan, int reps, fls_stream_t stream);
/* Name of the variant segment 0 / 1 of the plan launches ("" when the plan has no such segment). */
const char* fls_plan_variant_name(const fls_plan* plan, int segment);
/* fls_plan_decode through a CUDA graph: the plan's launches (one per kernel family its queue holds) are
 * captured once, on the first call or the first after fls_plan_autotune, and replayed on `stream`. */
int fls_plan_decode_graph(fls_plan* plan, fls_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Reference page columns on the device.  d_page holds the bytes of one FastLanes page (the data_buf of
 * ExpColEncoder, src/encoder/exp_col_encoder.cpp:40-64); d_dict the dictionary bytes for DICT / DICT_RLE
 * expressions.  Replaces TColDecoder::{ExtInitDict, InitDecompress, Decompress} plus the materialisation of
 * include/fls/encoder/assert_eq.hpp:50-400 for the integer expressions: UNCOMPRESSED, FFOR, DELTA, RLE
 * (UNCOMPRESSED / DELTA_NO_PATCH), DICT (UNCOMPRESSED / FFOR / DELTA), DICT_RLE (UNCOMPRESSED / DELTA).
 * d_page may sit at any byte address and d_out must be 16-byte aligned; a packed buffer that starts 16-byte
 * aligned is staged by TMA (fls_page_placement gives the shift that achieves it), any other by the warp.
 * Several columns decode in one launch.
 * ------------------------------------------------------------------------------------------------------- */
typedef struct {
	const uint8_t* d_page;
	uint64_t       page_size;
	const uint8_t* d_dict; /* NULL unless the expression has a dictionary */
	uint64_t       dict_size;
	uint8_t        data_type; /* enum data_t of fastlanes.h: INT64, UINT64, INT32, UINT32, INT16, UINT16, DOUBLE
	                             (bit patterns; a DOUBLE dictionary page holds its values raw) */
	uint8_t        order;     /* fls_order_code; FLS_ORIGINAL is what the reference materialises */
	uint8_t        reserved[6];
	void*          d_out; /* vec_c * 1024 values of data_type */
} fls_page_column;

/* Header facts of a page from its first bytes (prefix_size >= 8 + 4 * arr_c). */
int fls_page_info(const uint8_t* page_prefix, uint64_t prefix_size, uint32_t* exp_t, uint32_t* var, uint32_t* vec_c,
                  uint32_t* arr_c, uint64_t* meta_size);
/* Byte shift (0..15) to add to a 16-byte aligned device address so that the page's packed buffer lands on a
 * 16-byte boundary. */
int fls_page_placement(const uint8_t* page_prefix, uint64_t prefix_size, uint32_t* shift);
int fls_gpu_decode_pages(const fls_page_column* cols, uint32_t n_cols, fls_stream_t stream);
/* Random access by vector: vectors [first_vec, first_vec + n_vec) of one page, vector first_vec + i written at
 * col->d_out + i * 1024 values (the reference's Reader::get_chunk, src/reader/reader.cpp:19-61, and the
 * random_access it declares but never defines, include/fastlanes.h:88-106).  Page-wide buffers (rec buffers,
 * a patched DICT's code stream) are decoded whole; FLS_ERR_ARG for a range past the page's vectors. */
int fls_gpu_decode_page_vectors(const fls_page_column* col, uint32_t first_vec, uint32_t n_vec, fls_stream_t stream);
/* fls_gpu_decode_pages reads each page header in stream order on `stream` (it synchronises that stream once).
 * The same decode as a plan: page metadata is read once here (on the legacy default stream, so the pages must
 * already be in place); fls_plan_decode then only launches.  Replaces
 * the reference's per-vector page walk (Page::InitDecompress + page_params, src/cor/lyt/page/page.cpp:63-139). */
int fls_plan_create_pages(const fls_page_column* cols, uint32_t n_cols, fls_plan** out_plan);

/* ---------------------------------------------------------------------------------------------------------
 * Predicate pushdown on compressed columns.  Replaces the reference's per-vector predicate primitives on
 * decoded i64 vectors (src/primitive/predicate/equal.cpp:9-99: eq_vector_constant_func, ge_tvec_cvec,
 * lessthan_func, behind predicate_eq_vector_constant_i64 / predicate_GT_i64 / predicate_LE_i64 of
 * include/fls/expression/predicate_operator.hpp:7-112) and and_selection_ds_func (equal.cpp:100-119), for every
 * integer expression and type the page decoder handles.  The values are decoded in registers and never
 * written: each vector yields a 1024-bit bitmap (16 u64 words, the layout of SelectionDS::bitmap,
 * include/fls/expression/selection_ds.hpp:27), bit i = value i of the vector in the column's order.  Note the
 * reference's operators: predicate_GT_i64 computes `>`, predicate_LE_i64 computes `<` (lessthan_func).
 * ------------------------------------------------------------------------------------------------------- */
#define FLS_PRED_EQ 0 /* value == constant */
#define FLS_PRED_NE 1
#define FLS_PRED_LT 2 /* value <  constant (the reference's predicate_LE_i64 / lessthan_func) */
#define FLS_PRED_LE 3
#define FLS_PRED_GT 4 /* value >  constant (the reference's predicate_GT_i64 / ge_tvec_cvec) */
#define FLS_PRED_GE 5
typedef struct {
	uint8_t op; /* FLS_PRED_* */
	uint8_t reserved[7];
	int64_t value; /* the constant; compared with each value widened to 64 bits: sign-extended for the signed
	                  data types (value read as int64), zero-extended for the unsigned ones (value read as its
	                  uint64 bits) */
} fls_predicate;
/* A filter plan over page columns (as fls_plan_create_pages; DOUBLE columns are refused): cols[i].d_out
 * receives vec_c * 128 bytes, one bitmap per vector; fls_plan_decode / fls_plan_decode_graph evaluate. */
int fls_plan_create_filter(const fls_page_column* cols, uint32_t n_cols, const fls_predicate* pred,
                           fls_plan** out_plan);
/* SelectionDS::idx_arr / n_selected_values per vector from bitmaps (equal.cpp:12-28, the index form):
 * d_idx: n_vec * 1024 u16 positions in ascending order (entries past the count are left as they are),
 * d_count: n_vec u16.  Asynchronous. */
int fls_gpu_bitmap_to_selection(const uint64_t* d_bitmaps, uint64_t n_vec, uint16_t* d_idx, uint16_t* d_count,
                                fls_stream_t stream);
#define FLS_BITMAP_AND 0
#define FLS_BITMAP_OR 1
#define FLS_BITMAP_ANDNOT 2 /* a & ~b */
/* Word-wise combination of n_vec bitmaps (d_out may alias an input). */
int fls_gpu_bitmap_combine(const uint64_t* d_a, const uint64_t* d_b, uint64_t* d_out, uint64_t n_vec, int op,
                           fls_stream_t stream);
/* and_selection_ds_func (equal.cpp:100-119) per vector: the positions present in both index lists (each
 * ascending, positions < 1024), ascending.  Lists of d_count0 / d_count1 entries at d_idx0 / d_idx1 + 1024 * v;
 * an out-of-range position or count sets FLS_DEV_BAD_INDEX (fls_gpu_status). */
int fls_gpu_selection_and(const uint16_t* d_idx0, const uint16_t* d_count0, const uint16_t* d_idx1,
                          const uint16_t* d_count1, uint16_t* d_idx_out, uint16_t* d_count_out, uint64_t n_vec,
                          fls_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Files: the reference's file pair data.fls + footer.json, written by Connection::to_fls (src/connection.cpp:
 * 102-128) and opened by Connection::read_fls / Reader (src/reader/reader.cpp:19-61), read into device memory.
 * Footer keys as src/json/fls_json.cpp:30-62 writes them.  The reference stores values only for its
 * ZERO_COPY columns (n_vec * 1024 raw values at col_ofs); for CONSTANT / EQUAL columns it keeps neither the
 * constant nor the equal column's index, so they report FLS_FILE_NO_DATA.  Page columns (FLS_FILE_PAGES) are
 * this library's extension of the same container: a "pages" list of row-group chunks of reference page bytes
 * ({"ofs", "size", "dict_ofs", "dict_size", "n_vec"}), decoded on the GPU.
 * ------------------------------------------------------------------------------------------------------- */
#define FLS_FILE_ZERO_COPY 1
#define FLS_FILE_PAGES 2
#define FLS_FILE_NO_DATA 3
typedef struct fls_file fls_file;
/* Parses dir/footer.json and checks the column ranges against dir/data.fls (host only, no GPU work). */
int fls_file_open(const char* dir, fls_file** out_file);
int fls_file_shape(const fls_file* file, uint32_t* n_cols, uint64_t* n_vec);
/* data_type: enum data_t of fastlanes.h; kind: FLS_FILE_*; n_values: values a read writes (0 for NO_DATA). */
int fls_file_column(const fls_file* file, uint32_t col, uint8_t* data_type, uint8_t* kind, uint64_t* n_values);
/* Reads columns cols[0..n) into d_outs[i] (n_values values each, original order, 16-byte aligned): the file's
 * bytes stream through two pinned bounce buffers (the read of one overlapping the copy out of the other);
 * ZERO_COPY columns land directly in their outputs, the chunks of every page column are staged and decoded by
 * one page decode.  FLS_ERR_UNSUPPORTED for a NO_DATA column.  Synchronous. */
int fls_file_read(fls_file* file, const uint32_t* cols, uint32_t n, void* const* d_outs, fls_stream_t stream);
int fls_file_close(fls_file* file);

/* ---------------------------------------------------------------------------------------------------------
 * String columns.  d_page: a string page (BYTE_ARR: str expressions 0, 1; DICT: 2-12; FSST: 13, 14;
 * DICT_RLE: 15, 16; DICT_FRQ: 17-27; FSST12: 28, 29 of src/cor/exp_pool.cpp:66-101); d_dict: its dictionary
 * bytes (DICT / DICT_RLE / DICT_FRQ: the FSST-compressed dictionary page; FSST / FSST12: the exported symbol
 * table; BYTE_ARR: none).  Creating a plan decodes the
 * dictionary once on the GPU (TColDecoder::ExtInitDict, src/encoder/col_encoder.cpp:198-201); decoding emits
 * Arrow-style output: n_rows + 1 u32 offsets and the concatenated bytes, rows in original order
 * (include/fls/encoder/assert_eq.hpp:166-210, :257-400).  The page and dictionary buffers must outlive the plan.
 * Device memory a plan holds: 16 bytes per vector, the decoded dictionary (DICT kinds), a decoded code stream
 * of 4 bytes per row (DICT pages with patched codes) or every row's decoded length, 4 bytes per row (FSST12
 * pages).
 * ------------------------------------------------------------------------------------------------------- */
typedef struct fls_string_plan fls_string_plan;
int fls_string_plan_create(const uint8_t* d_page, uint64_t page_size, const uint8_t* d_dict, uint64_t dict_size,
                           fls_string_plan** out_plan);
int fls_string_plan_rows(const fls_string_plan* plan, uint64_t* n_rows);
/* Total decoded bytes (runs the length pass; synchronises the stream). */
int fls_string_plan_measure(fls_string_plan* plan, uint64_t* n_bytes, fls_stream_t stream);
/* d_offsets: n_rows + 1 entries; d_bytes: 16-byte aligned, bytes_cap < 4 GiB.  Asynchronous, no allocation.
 * FSST and BYTE_ARR pages, and DICT pages whose dictionary entries are < 256 bytes, decode in one launch (after
 * one memset): every vector finds its first output byte by a look-back over the earlier vectors' totals.  Other
 * pages (FSST12, DICT with longer entries) run the length pass themselves unless a measure() came just before
 * (whose totals they then take over).  The plan keeps that scratch (look-back words, totals), so decodes of one
 * plan whose work overlaps on the GPU (other streams) race: order them, or give each stream its own plan. */
int fls_string_plan_decode(const fls_string_plan* plan, uint32_t* d_offsets, uint8_t* d_bytes, uint64_t bytes_cap,
                           fls_stream_t stream);
int fls_string_plan_destroy(fls_string_plan* plan);

/* ---------------------------------------------------------------------------------------------------------
 * String sets: many DICT string columns (string pool DICT / DICT_RLE / DICT_FRQ pages, each with its own
 * FSST-compressed dictionary whose entries are < 256 bytes) decoded by ONE kernel launch (after one memset of the
 * set's scratch), the multi-column form of fls_string_plan_decode for a row group's string columns
 * (the reference decodes them column by column: TColDecoder<str_pt>, src/encoder/col_encoder.cpp:198-217).
 * create: from plans made by fls_string_plan_create (they must outlive the set; FLS_ERR_UNSUPPORTED for a plan of
 *   another kind).  bind: each column's outputs (as fls_string_plan_decode's: n_rows + 1 u32 offsets, 16-byte
 *   aligned bytes, capacity < 4 GiB); synchronous, once.  decode: asynchronous, no allocation, capturable in a
 *   CUDA graph; decodes of one set whose work overlaps on the GPU race on its scratch.  Device memory a set
 *   holds: 8 bytes per vector and per CTA-sized chunk of vectors.
 * ------------------------------------------------------------------------------------------------------- */
typedef struct fls_string_set fls_string_set;
int fls_string_set_create(const fls_string_plan* const* plans, uint32_t n, fls_string_set** out_set);
int fls_string_set_bind(fls_string_set* set, uint32_t* const* d_offsets, uint8_t* const* d_bytes,
                        const uint64_t* bytes_caps);
int fls_string_set_decode(const fls_string_set* set, fls_stream_t stream);
int fls_string_set_destroy(fls_string_set* set);

/* Allocation-free decode of an FSST (str expressions 13, 14) or BYTE_ARR (0) page.  No counterpart in the
 * reference.  Some callers cannot allocate device memory: an engine whose buffer manager owns all of HBM and
 * forbids plugins to call cudaMalloc, or a caller on a path where allocating is not allowed.  This call needs no
 * allocation: its scratch (per-vector byte totals and bases, the FSST table) is one fixed array of
 * FLS_NOALLOC_SCRATCH_BYTES compiled into the library, which every GPU that loads the library holds until the
 * process exits, and it never touches the library's per-device state (which is allocated on first use).
 * Limits and rules:
 *   - at most FLS_NOALLOC_MAX_VECTORS vectors (8,388,608 rows) per page; larger pages return FLS_ERR_TOO_LARGE
 *     before any work;
 *   - the first call on a device looks up the array's device address (cudaGetSymbolAddress);
 *   - every call reads the page header and the symbol table back to the host in `stream`'s order (after the
 *     work queued on it before) and waits for those reads;
 *   - all calls share the array, so calls whose work overlaps on the GPU (other streams, other threads) race;
 *     serialise them;
 *   - d_status is required (FLS_ERR_ARG when null): device-detected errors (FLS_DEV_*) are OR-ed into it, and
 *     the caller zeroes it before the call.
 * Inputs and outputs are as for fls_string_plan_decode: d_offsets n_rows + 1 u32, d_bytes 16-byte aligned with
 * room for the decoded bytes (bytes_cap < 4 GiB); d_dict holds the FSST table bytes for FSST pages. */
#define FLS_NOALLOC_MAX_VECTORS 8192
#define FLS_NOALLOC_SCRATCH_BYTES 133392
int fls_gpu_decode_fsst_page_noalloc(const uint8_t* d_page, uint64_t page_size, const uint8_t* d_dict,
                                     uint64_t dict_size, uint32_t* d_offsets, uint8_t* d_bytes, uint64_t bytes_cap,
                                     int* d_status, fls_stream_t stream);

/* ---------------------------------------------------------------------------------------------------------
 * Encoders for string pages (host memory in and out).
 * fls_fsst_compress: builds an FSST symbol table over n strings (Arrow offsets, n + 1) and compresses them;
 *   table_out receives the table in fsst_export's format (src/cor/prm/fsst/libfsst.cpp:581-615, read by
 *   fsst_import :617-657), comp_offsets (n + 1) the compressed strings' boundaries.
 * fls_encode_string_dict: a string DICT FFOR_NO_PATCH page (str expression 3, src/cor/exp_pool.cpp:69) of
 *   n_rows codes into a dictionary of n_dict strings, and its FSST-compressed dictionary page
 *   (src/cor/lyt/dic/dic.cpp:88-111) with the true compressed length of every entry.
 * ------------------------------------------------------------------------------------------------------- */
int fls_fsst_compress(const uint8_t* bytes, const uint64_t* offsets, uint64_t n, uint8_t* table_out,
                      uint64_t table_cap, uint64_t* table_size, uint8_t* comp_out, uint64_t comp_cap,
                      uint64_t* comp_offsets);
int fls_encode_string_dict(const uint8_t* dict_bytes, const uint64_t* dict_offsets, uint32_t n_dict,
                           const uint32_t* codes, uint64_t n_rows, uint8_t* page_out, uint64_t page_cap,
                           uint64_t* page_size, uint8_t* dict_out, uint64_t dict_cap, uint64_t* dict_size);

/* DICT / DICT_RLE encoding of an integer column of width 32 or 64 (host memory, whole vectors of n): the
 * dictionary page (dict_hdr_t + a rec buffer holding the entries raw, first-occurrence order as
 * src/cor/lyt/dic/dic_fac.cpp:19-40 assigns them) and the codes page, DICT FFOR_NO_PATCH (exp 8 var 2, int
 * pool id 17) or with rle = 1 DICT_RLE DELTA_NO_PATCH (exp 11 var 2: the RLE layout over u32 run codes; the
 * int pool's id 27 additionally packs the run codes).  *page_size / *dict_size receive the sizes. */
int fls_encode_int_dict(const void* in, uint64_t n, int width, int rle, uint8_t* page_out, uint64_t page_cap,
                        uint64_t* page_size, uint8_t* dict_out, uint64_t dict_cap, uint64_t* dict_size);

#ifdef __cplusplus
}
#endif
#endif /* FLS_B200_H */
