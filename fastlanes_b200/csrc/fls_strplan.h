// Arguments of the string kernels (shared by the host string plan and fls_k_strings.cu).
#pragma once

#include "fls_plan.h"
#include <cstdint>
#include <cuda_runtime.h>

namespace flsgpu {

// FSST symbol table as the decoder uses it: symbol c (little-endian) and its length.
struct FsstTable {
	uint64_t sym[256];
	uint8_t  len[256];
};

// FSST12 symbol table (include/fls/cor/prm/fsst12/fsst12.h:74-79): 4096 codes of 12 bits, symbol c
// (little-endian) and its length.
struct Fsst12Table {
	uint64_t sym[4096];
	uint8_t  len[4096];
};

enum : uint8_t {
	STR_DICT  = 0, // rows are dictionary codes (DICT / DICT_RLE pages), dictionary FSST-decoded once per plan
	STR_FSST  = 1, // rows are FSST-compressed in the page (FSST pages)
	STR_BYTES = 2, // rows are plain bytes in the page (BYTE_ARR pages)
	STR_FSST12 = 3, // rows are FSST12-compressed in the page (FSST12 pages)
};

constexpr int      kStrMaxWarps   = 32;        // warps per CTA of the string kernels (at most)
constexpr int      kStrLenWarps   = 16;        // warps per CTA of the lengths pass
constexpr uint32_t kStrEndsSmemMax = 64 * 1024; // largest dictionary end-offset array copied to shared memory
// static shared memory of the FSST12 string kernels (the symbol table), taken from the dynamic budget
constexpr uint32_t kStrFsst12Smem = sizeof(Fsst12Table);

struct StrArgs {
	ColDesc          col; // the row stream: codes or cumulative end offsets, page layout
	uint8_t          kind;
	bool             dict_in_smem; // materialising pass: decoded dictionary bytes in shared memory
	bool             ends_in_smem; // lengths pass: dictionary end offsets in shared memory
	bool             rows16;       // DICT with fewer than 65535 entries: codes kept as 16-bit rows
	uint32_t         entry_c;
	const uint32_t*  dict_ends;
	// materialising pass: entry c as start | length << 24 (dictionaries of < 16 MiB decoded bytes whose
	// entries are all < 256 bytes), one load per row instead of two end offsets; null otherwise
	const uint32_t*  dict_rows;
	// FSST12 pages: every row's decoded length, written by the lengths pass and read by the materialising pass
	// instead of walking the row's codes a second time (null: both walk them)
	uint32_t*        row_len;
	const uint8_t*   dict_bytes;
	uint64_t         dict_bytes_n;
	const FsstTable* table;
	const Fsst12Table* table12; // FSST12 pages
	uint64_t*        vec_total;
	const uint64_t*  vec_base;
	uint32_t*        offsets;
	uint8_t*         bytes;
	uint64_t         bytes_cap;
	int*             status;
	uint64_t         item_base; // single-pass DICT decode: index of the column's vector 0 among the look-back words
};

// One launch of the single-pass DICT decode (k_dict_pass) over the vectors of one or more DICT string columns.
// Work is taken in chunks of chunk_w vectors of one column (a chunk per CTA, by an atomic ticket); every vector
// publishes its decoded byte total and, once its predecessors' totals are known, its inclusive prefix (a
// decoupled look-back within its column), so each vector learns its first output byte without a separate
// lengths pass.
struct StrSetArgs {
	const StrArgs*  cols;      // per-column arguments in device memory (each with dict_rows: start | length << 24)
	const uint32_t* chunk_col; // column of every chunk (null: one column, chunk c = its vectors [c * chunk_w, ...))
	const uint32_t* chunk_v0;  // first vector of every chunk (null: as above)
	uint32_t        n_chunks;
	uint32_t        chunk_w;   // vectors per chunk = warps per CTA
	uint64_t*       flags;     // [0] the chunk ticket, [1 + item_base + v] the look-back word of vector v; zeroed
	                           // before every launch
	int*            status;
	uint32_t*       out_offsets; // one-column launches: the outputs (null: each column's own)
	uint8_t*        out_bytes;
	uint64_t        out_cap;
	uint32_t        dict_cap; // shared memory held for a dictionary's bytes (16-byte multiple; 0: dictionaries in
	                          // global memory)
	uint32_t        tab_cap;  // entries held for the packed row table (with dict_cap)
};

// per-warp shared memory of k_dict_pass: the vector's rows and the output window
uint32_t dict_pass_smem_per_warp(bool rows16);
cudaError_t launch_dict_pass(const StrSetArgs& a, bool rows16, int warps, uint32_t dyn_smem, cudaStream_t s,
                             int sm_count = 0);

cudaError_t launch_fsst_dict(const uint8_t* lens, const uint8_t* comp, uint64_t comp_size, uint32_t entry_c,
                             const FsstTable* tab, uint32_t* ends, uint8_t* bytes, uint64_t cap, int* status,
                             cudaStream_t s);
// sm_count: the device's SM count, or 0 to take it from the library's per-device state (current_device())
cudaError_t launch_str_lengths(const StrArgs& a, int sm_count, cudaStream_t s);
// Single-pass FSST / BYTE_ARR decode (k_stream_single): lb = a ticket word then one zeroed look-back word per
// vector; writes a.offsets / a.bytes (capacity a.bytes_cap).
cudaError_t launch_stream_single(const StrArgs& a, uint64_t* lb, cudaStream_t s, int sm_count = 0);
cudaError_t launch_scan_totals(const uint64_t* total, uint64_t* base, uint64_t n, cudaStream_t s);
// warps: warps per CTA (at most kStrMaxWarps); dyn_smem: warps * str_smem_per_warp(a.rows16) plus the
// 16-byte rounded dictionary bytes when a.dict_in_smem
cudaError_t launch_str_materialize(const StrArgs& a, int warps, uint32_t dyn_smem, cudaStream_t s, int sm_count = 0);
uint32_t    str_smem_per_warp(bool rows16);
// shared-memory bytes of the dictionary end offsets (16-byte rounded)
__host__ __device__ inline uint32_t str_ends_smem(const StrArgs& a) { return (a.entry_c * 4u + 15u) & ~15u; }

} // namespace flsgpu
