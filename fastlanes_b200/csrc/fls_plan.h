// Column descriptors shared by the host runtime (C++) and the decode kernels (CUDA).
//
// A decode launch walks a queue of (column, vector) work items.  Each column says how its 1024-value vectors
// are stored: either as plain per-vector arrays (the primitive API: packed words + bw + base arrays) or as a
// FastLanes page (PageHdr + buffer offsets + entry points + buffers, src/cor/eng/compressor.cpp:68-86 and
// src/cor/lyt/page/page.cpp:63-139 of the reference), and what the decoded stream turns into
// (plain values, RLE expansion, dictionary gather).
#pragma once

#include <cstdint>

namespace flsgpu {

enum : uint8_t {
	ENC_RAW   = 0, // 1024 transposed values stored verbatim (bw = W)
	ENC_FFOR  = 1, // bit-packed, plus FOR base
	ENC_DELTA = 2, // bit-packed deltas + FOR base, then per-lane running sum from 128-byte lane bases
};

enum : uint8_t {
	POST_NONE     = 0, // output = decoded stream
	POST_RLE      = 1, // stream is a u16 run index; output = run_values[index]
	POST_DICT     = 2, // stream is u32 codes; output = dict[code]
	POST_RLE_DICT = 3, // stream is a u16 run index into u32 codes; output = dict[codes[index]]
	// patched FFOR / DELTA: the unpacked values (transposed positions) are patched before rsum
	// (src/cor/prm/patch/*_decompress.cpp)
	POST_PATCH_S  = 4, // exceptions + (exc_c u16, exc_c u16 positions)
	POST_PATCH_B  = 5, // exceptions + 1024-bit position bitmap (16 u64 words), exceptions in bit order
	POST_PATCH_LL = 6, // exceptions + (exc_c u16, first position u16); gaps chained through the packed values
};

// RLE / DICT gathers read a second array per value (gather kernels); patches stay in the plain kernels.
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr bool post_is_gather(uint32_t post) { return post >= POST_RLE && post <= POST_RLE_DICT; }
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr bool post_is_patch(uint32_t post) { return post >= POST_PATCH_S && post <= POST_PATCH_LL; }

enum : uint8_t {
	LAYOUT_ARRAYS = 0,
	LAYOUT_PAGE   = 1,
};

constexpr uint8_t kNoBuf = 0xFF;

struct alignas(16) ColDesc {
	// what
	uint8_t  ws;     // stream width in bits: 8, 16, 32, 64
	uint8_t  e;      // output element size in bytes: 1, 2, 4, 8
	uint8_t  enc;    // ENC_*
	uint8_t  post;   // POST_*
	uint8_t  order;  // 0 transposed (primitive order), 1 original (materialised)
	uint8_t  layout; // LAYOUT_*
	uint8_t  arr_c;  // page: number of buffers
	uint8_t  bw_const;
	uint32_t n_vec;
	uint32_t entry_c; // dictionary entries (POST_DICT / POST_RLE_DICT)

	// LAYOUT_PAGE: role -> buffer index (kNoBuf when absent) and resolved buffer starts
	uint8_t  ib_bw, ib_base, ib_packed, ib_lane_bases, ib_vals;
	uint8_t  ib_exc, ib_side; // patched variants: exception values, positions / bitmap / chain head
	uint8_t  out_mode;        // OUT_VALUES, or OUT_BITMAP_*: `out` takes one 1024-bit predicate bitmap per vector
	const uint8_t*  buf[6];
	uint64_t        buf_size[6];
	const uint32_t* ep; // entry points, (n_vec - 1) x arr_c u32; vector 0 starts at 0 in every buffer

	// LAYOUT_ARRAYS
	const uint8_t*  packed;     // packed words of all vectors
	const uint64_t* byte_off;   // per-vector byte offset into packed; null => v * bw_const * 128
	const uint8_t*  bw_arr;     // per-vector bit width; null => bw_const
	const uint8_t*  base_arr;   // per-vector FOR base (ws/8 bytes each); null => 0
	const uint8_t*  lane_base_arr; // per-vector 128-byte lane bases (ENC_DELTA)

	// gathers and output
	const uint8_t* dict; // POST_DICT: entry_c values of e bytes
	uint8_t*       out;  // n_vec * 1024 * e bytes (OUT_VALUES) or n_vec * 128 bytes (bitmaps)
};

enum : uint8_t {
	OUT_VALUES   = 0,
	OUT_BITMAP_U = 1, // bitmap of `value OP constant`, values compared as unsigned e-byte integers
	OUT_BITMAP_S = 2, // the same, values compared as signed (two's complement) e-byte integers
};

// Predicate of a filter launch: value OP constant, the constant widened to 64 bits (sign-extended for signed
// columns).  Mirrors the reference's predicate primitives (src/primitive/predicate/equal.cpp).
enum : uint32_t { PRED_EQ = 0, PRED_NE = 1, PRED_LT = 2, PRED_LE = 3, PRED_GT = 4, PRED_GE = 5 };
struct Pred {
	uint64_t value;
	uint32_t op;
	uint32_t active; // nonzero: the launch is a filter (KIND_FILTER kernels of the segment's family)
};

struct DecodeArgs {
	const ColDesc*  cols;   // device array of columns, or null => use col0
	const uint32_t* queue;  // device array of (col << col_shift | vec) items, or null => vectors of col0
	uint64_t        n_items;
	int*            status;    // device word; kernels OR error bits into it
	uint32_t        col_shift; // 24 for batch plans (256 batches), 16 for page plans (65,535 pages)
	ColDesc         col0;
	Pred            pred; // filter launches (KIND_FILTER kernels) only
	// failure injection (fls_gpu_test_stalled_copy only; 0 otherwise): work item test_stall - 1 arms its copies'
	// byte count without issuing them, so nothing is in flight and its wait runs out; spin_limit bounds the
	// decode loop's waits (0: kMbarSpinLimit)
	uint64_t        test_stall;
	uint32_t        spin_limit;
};

enum : int {
	STATUS_TIMEOUT    = 1,  // an mbarrier wait hit its bound
	STATUS_BAD_BW     = 2,  // bit width above the stream width
	STATUS_BAD_INDEX  = 4,  // RLE index or dictionary code out of range
	STATUS_BAD_LAYOUT = 8,  // page buffer reference outside the page
};

} // namespace flsgpu
