// Host side of the page path: reading FastLanes page metadata, mapping expressions onto the decode engine's
// column descriptors, and the reference's C API (include/fastlanes.h).
//
// Page bytes (src/cor/eng/compressor.cpp:68-86, src/cor/lyt/page/page.cpp:63-139,
// src/cor/lyt/page/entry_point.cpp:21-41, include/fls/cor/lyt/page/page_hdr.hpp:8-15):
//   [PageHdr 8 B: exp_t u8, var u8, reserved u16, vec_c u16, pad u16]
//   [arr_c x u32 absolute buffer offsets]
//   [(vec_c - 1) x arr_c x u32 entry points (vector 0 starts every buffer at 0)]
//   [buffer 0] ... [buffer arr_c - 1]
// The buffer roles per expression come from the compress RPN tables (include/fls/cor/exp/*/*_exp.hpp) and the
// compress primitives that fill them (src/cor/prm/{ffor,rsum,rle}/*_compress.cpp, src/cor/lyt/vec.cpp:40-120).
#include "fastlanes.h"
#include "fls_b200.h"
#include "fls_page.h"
#include "fls_rec.h"
#include "fls_runtime.h"

#include <algorithm>
#include <cstring>
#include <cuda_runtime.h>
#include <vector>

namespace flsgpu {

const ExprLayout* expr_layout(uint8_t exp_t, uint8_t var) {
	// exp_t, var, arr_c, stream width (0 = value width), enc, post, roles: bw, base, packed, lane, vals, rec buffer,
	// exceptions, positions
	constexpr uint8_t N = kNoBuf;
	static const ExprLayout table[] = {
	    {2, 1, 1, 0, ENC_RAW, POST_NONE, N, N, 0, N, N, N, N, N, 0},                     // UNCOMPRESSED
	    {4, 1, 3, 0, ENC_FFOR, POST_NONE, 0, 1, 2, N, N, N, N, N, 0},                    // FFOR NO_PATCH
	    {4, 2, 5, 0, ENC_FFOR, POST_PATCH_LL, 2, 3, 4, N, N, N, 0, 1, 0},                // FFOR LL_PATCH
	    {4, 3, 5, 0, ENC_FFOR, POST_PATCH_S, 2, 3, 4, N, N, N, 0, 1, 0},                 // FFOR S_PATCH
	    {4, 4, 5, 0, ENC_FFOR, POST_PATCH_B, 2, 3, 4, N, N, N, 0, 1, 0},                 // FFOR B_PATCH
	    {4, 5, 5, 0, ENC_FFOR, POST_PATCH_S, 2, 3, 4, N, N, 0, 0, 1, 0},                 // FFOR S_PATCH_REC
	    {5, 1, 4, 0, ENC_DELTA, POST_NONE, 1, 2, 3, 0, N, N, N, N, 0},                   // DELTA NO_PATCH
	    {5, 2, 6, 0, ENC_DELTA, POST_PATCH_LL, 3, 4, 5, 0, N, N, 1, 2, 0},               // DELTA LL_PATCH
	    {5, 3, 6, 0, ENC_DELTA, POST_PATCH_S, 3, 4, 5, 0, N, N, 1, 2, 0},                // DELTA S_PATCH
	    {5, 4, 6, 0, ENC_DELTA, POST_PATCH_B, 3, 4, 5, 0, N, N, 1, 2, 0},                // DELTA B_PATCH
	    {5, 5, 6, 0, ENC_DELTA, POST_PATCH_B, 3, 4, 5, 0, N, 1, 1, 2, 0},                // DELTA B_PATCH_REC
	    {6, 1, 2, 16, ENC_RAW, POST_RLE, N, N, 1, N, 0, N, N, N, 0},                     // RLE UNCOMPRESSED
	    {6, 2, 5, 16, ENC_DELTA, POST_RLE, 2, 3, 4, 1, 0, N, N, N, 0},                   // RLE DELTA_NO_PATCH
	    {6, 3, 2, 16, ENC_RAW, POST_RLE, N, N, 1, N, 0, 0, N, N, 0},                     // RLE UNCOMPRESSED_REC
	    {6, 4, 5, 16, ENC_DELTA, POST_RLE, 2, 3, 4, 1, 0, 0, N, N, 0},                   // RLE DELTA_NO_PATCH_REC
	    {6, 5, 5, 16, ENC_DELTA, POST_RLE, 2, 3, 4, 1, 0, 0, N, N, 0, 1},                // RLE DELTA_NO_PATCH_REC2
	    {8, 1, 1, 32, ENC_RAW, POST_DICT, N, N, 0, N, N, N, N, N, 0},                    // DICT UNCOMPRESSED
	    {8, 2, 3, 32, ENC_FFOR, POST_DICT, 0, 1, 2, N, N, N, N, N, 0},                   // DICT FFOR_NO_PATCH
	    {8, 7, 4, 32, ENC_DELTA, POST_DICT, 1, 2, 3, 0, N, N, N, N, 0},                  // DICT DELTA_NO_PATCH
	    // DICT with patched codes (dict_exp.hpp:31-41): the code stream laid out as the patched FFOR / DELTA pages
	    {8, 3, 5, 32, ENC_FFOR, POST_PATCH_LL, 2, 3, 4, N, N, N, 0, 1, 1},            // DICT FFOR_LL_PATCH
	    {8, 4, 5, 32, ENC_FFOR, POST_PATCH_S, 2, 3, 4, N, N, N, 0, 1, 1},             // DICT FFOR_S_PATCH
	    {8, 5, 5, 32, ENC_FFOR, POST_PATCH_B, 2, 3, 4, N, N, N, 0, 1, 1},             // DICT FFOR_B_PATCH
	    {8, 6, 5, 32, ENC_FFOR, POST_PATCH_S, 2, 3, 4, N, N, 0, 0, 1, 1},             // DICT FFOR_S_PATCH_REC
	    {8, 8, 6, 32, ENC_DELTA, POST_PATCH_LL, 3, 4, 5, 0, N, N, 1, 2, 1},           // DICT DELTA_LL_PATCH
	    {8, 9, 6, 32, ENC_DELTA, POST_PATCH_S, 3, 4, 5, 0, N, N, 1, 2, 1},            // DICT DELTA_S_PATCH
	    {8, 10, 6, 32, ENC_DELTA, POST_PATCH_B, 3, 4, 5, 0, N, N, 1, 2, 1},           // DICT DELTA_B_PATCH
	    {8, 11, 6, 32, ENC_DELTA, POST_PATCH_B, 3, 4, 5, 0, N, 1, 1, 2, 1},           // DICT DELTA_B_PATCH_REC
	    {11, 1, 2, 16, ENC_RAW, POST_RLE_DICT, N, N, 1, N, 0, N, N, N, 0},               // DICT_RLE UNCOMPRESSED
	    {11, 2, 5, 16, ENC_DELTA, POST_RLE_DICT, 2, 3, 4, 1, 0, N, N, N, 0},             // DICT_RLE DELTA_NO_PATCH
	    {11, 3, 2, 16, ENC_RAW, POST_RLE_DICT, N, N, 1, N, 0, 0, N, N, 0},               // DICT_RLE UNCOMPRESSED_REC
	    {11, 4, 5, 16, ENC_DELTA, POST_RLE_DICT, 2, 3, 4, 1, 0, 0, N, N, 0},             // DICT_RLE ..._REC
	};
	// DICT_FRQ (exp_t 9) pages are DICT pages: dict_frq_exp derives dict_exp (dict_exp.hpp:208), only the
	// dictionary's order differs (frequency instead of first occurrence)
	const uint8_t et = exp_t == 9 ? 8 : exp_t;
	for (const auto& e : table) {
		if (e.exp_t == et && e.var == var) { return &e; }
	}
	return nullptr;
}

int value_width_of(uint8_t data_type) {
	switch (data_type) {
	case INT64:
	case UINT64:
	case DOUBLE: return 64;
	case INT32:
	case UINT32: return 32;
	case INT16:
	case UINT16: return 16;
	case INT8:
	case UINT8: return 8;
	default: return 0;
	}
}

int parse_page_header(const uint8_t* hdr, uint64_t avail, PageInfo* out) {
	if (avail < 8) { return FLS_ERR_FORMAT; }
	PageInfo pi {};
	pi.exp_t = hdr[0];
	pi.var   = hdr[1];
	std::memcpy(&pi.vec_c, hdr + 4, 2);
	pi.layout = expr_layout(pi.exp_t, pi.var);
	if (!pi.layout) { return FLS_ERR_UNSUPPORTED; }
	pi.arr_c = pi.layout->arr_c;
	if (avail < 8ull + 4ull * pi.arr_c) { return FLS_ERR_FORMAT; }
	for (uint32_t i = 0; i < pi.arr_c; ++i) { std::memcpy(&pi.off[i], hdr + 8 + 4 * i, 4); }
	pi.ep_off  = 8 + 4 * pi.arr_c;
	pi.meta_sz = pi.ep_off + 4ull * pi.arr_c * (pi.vec_c ? pi.vec_c - 1 : 0);
	*out       = pi;
	return FLS_OK;
}

int finish_page_info(PageInfo* pi, uint64_t page_size) {
	if (pi->vec_c == 0) { return FLS_OK; }
	if (pi->meta_sz > page_size) { return FLS_ERR_FORMAT; }
	for (uint32_t i = 0; i < pi->arr_c; ++i) {
		const uint64_t end = (i + 1 < pi->arr_c) ? pi->off[i + 1] : page_size;
		if (pi->off[i] < pi->meta_sz || pi->off[i] > end || end > page_size) { return FLS_ERR_FORMAT; }
		pi->size[i] = end - pi->off[i];
	}
	return FLS_OK;
}

int build_page_column(const PageInfo& pi, const uint8_t* d_page, int value_width, const uint8_t* d_dict_vals,
                      uint32_t dict_entries, int order, uint8_t* d_out, ColDesc* c, const uint8_t* d_vals_decoded,
                      uint64_t vals_decoded_size, const uint8_t* d_rec2, uint64_t rec2_size) {
	const ExprLayout* L = pi.layout;
	if (!L || value_width == 0) { return FLS_ERR_UNSUPPORTED; }
	// the page-level rec buffer of the _REC variants is decoded by the caller (rec_decode)
	if (L->ib_rec != kNoBuf && !d_vals_decoded) { return FLS_ERR_UNSUPPORTED; }
	if (L->ib_rec2 != kNoBuf && !d_rec2) { return FLS_ERR_UNSUPPORTED; }
	*c        = ColDesc {};
	c->ws     = static_cast<uint8_t>(L->ws ? L->ws : value_width);
	c->e      = static_cast<uint8_t>(value_width / 8);
	c->enc    = L->enc;
	c->post   = L->post;
	c->order  = static_cast<uint8_t>(order);
	c->layout = LAYOUT_PAGE;
	c->arr_c  = static_cast<uint8_t>(pi.arr_c);
	c->n_vec  = pi.vec_c;
	c->ib_bw  = L->ib_bw;
	c->ib_base = L->ib_base;
	c->ib_packed = L->ib_packed;
	c->ib_lane_bases = L->ib_lane;
	c->ib_vals = L->ib_vals;
	c->ib_exc  = L->ib_exc;
	c->ib_side = L->ib_side;
	for (uint32_t i = 0; i < pi.arr_c; ++i) {
		c->buf[i]      = d_page + pi.off[i];
		c->buf_size[i] = pi.size[i];
	}
	if (L->ib_rec != kNoBuf) {
		c->buf[L->ib_rec]      = d_vals_decoded;
		c->buf_size[L->ib_rec] = vals_decoded_size;
	}
	if (L->ib_rec2 != kNoBuf) {
		c->buf[L->ib_rec2]      = d_rec2;
		c->buf_size[L->ib_rec2] = rec2_size;
	}
	c->ep  = reinterpret_cast<const uint32_t*>(d_page + pi.ep_off);
	c->out = d_out;
	if (L->post == POST_DICT || L->post == POST_RLE_DICT) {
		if (!d_dict_vals || dict_entries == 0) { return FLS_ERR_FORMAT; }
		c->dict    = d_dict_vals;
		c->entry_c = dict_entries;
	}
	return FLS_OK;
}

int int_dictionary_values(const uint8_t* dict, uint64_t dict_size, int value_width, uint64_t* vals_off,
                          uint32_t* entries) {
	// only the first 20 bytes of dict are read; dict_size bounds the values
	// dict_hdr_t {exp_t u8, emp u8, emp u8, version u8, entry_c u32} (include/fls/cor/lyt/dic/dic.hpp:32-41)
	// followed by the dictionary values as a rec buffer (src/cor/lyt/dic/dic.cpp:142-144); rec_hdr
	// {bw u8, pad u8, exc_c u16, base[8]} (include/fls/cor/lyt/rec_hdr.hpp:7-13).  The raw form (bw = 255,
	// byte count in base) is a zero-copy view; FFOR blocks are not on this path.
	if (dict_size < 8 + 12) { return FLS_ERR_FORMAT; }
	uint32_t entry_c = 0;
	std::memcpy(&entry_c, dict + 4, 4);
	if (dict[8] != 255) { return FLS_ERR_UNSUPPORTED; }
	uint64_t raw = 0;
	std::memcpy(&raw, dict + 12, 8);
	const uint64_t need = static_cast<uint64_t>(entry_c) * (value_width / 8);
	if (raw != need || 20 + raw > dict_size) { return FLS_ERR_FORMAT; }
	*vals_off = 20;
	*entries  = entry_c;
	return FLS_OK;
}

} // namespace flsgpu

#ifndef FLS_HOST_EMULATION
// =========================================================================================================
// C ABI: page columns
// =========================================================================================================
using namespace flsgpu;

extern "C" {

int fls_page_info(const uint8_t* page_prefix, uint64_t prefix_size, uint32_t* exp_t, uint32_t* var,
                  uint32_t* vec_c, uint32_t* arr_c, uint64_t* meta_size) {
	PageInfo pi;
	const int rc = parse_page_header(page_prefix, prefix_size, &pi);
	if (rc != FLS_OK) { return rc; }
	if (exp_t) { *exp_t = pi.exp_t; }
	if (var) { *var = pi.var; }
	if (vec_c) { *vec_c = pi.vec_c; }
	if (arr_c) { *arr_c = pi.arr_c; }
	if (meta_size) { *meta_size = pi.meta_sz; }
	return FLS_OK;
}

// Descriptors, work queue and kernel family for a set of page columns.  Each page's header (and a dictionary's
// first 20 bytes) is read from the device in stream order on `stream`, so work queued before on that stream
// (e.g. the copy that brought the page in) is complete when the header is parsed.
static int read_on(void* dst, const void* src, size_t n, cudaStream_t stream) {
	if (cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, stream) != cudaSuccess) { return FLS_ERR_CUDA; }
	return cudaStreamSynchronize(stream) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

// Work items of page plans: (column << kPageShift | vector); a page holds at most 65,535 vectors.
constexpr uint32_t kPageShift = 16;

// Element bytes of a layout's rec-compressed buffer: run codes are idx_t = uint32, run values and exceptions
// the column's values.
static uint32_t rec_elem_bytes(const ExprLayout* L, int value_width) {
	return (L->post == POST_RLE_DICT || L->dict_codes) ? 4u : static_cast<uint32_t>(value_width / 8);
}

// Rec buffer at d_src (device, size bytes) decoded into a new device buffer, appended to *owned.
static int decode_rec_on(const uint8_t* d_src, uint64_t size, uint32_t eb, std::vector<void*>* owned,
                         const uint8_t** out, uint64_t* out_size, cudaStream_t stream) {
	std::vector<uint8_t> h(size);
	if (size && read_on(h.data(), d_src, size, stream) != FLS_OK) { return FLS_ERR_CUDA; }
	uint8_t*  buf = nullptr;
	const int rc  = rec_decode(d_src, h.data(), size, eb, &buf, out_size, stream);
	if (buf) { owned->push_back(buf); }
	*out = buf;
	return rc;
}

// col_desc (optional) receives, per column, the index of the descriptor that writes the column's output.  A
// DICT page with patched codes takes two descriptors: its patched code stream decoded into a buffer of the
// plan (in `owned`; a patched item, so it runs in an earlier launch segment than the gathers), then a raw
// 32-bit stream of those codes gathered from the dictionary.
extern "C++" {
namespace flsgpu {
int decode_patched_codes(const uint8_t* d_page, uint64_t page_size, uint32_t* d_codes, cudaStream_t stream) {
	uint8_t        hdr[8 + 4 * 8];
	const uint64_t take = page_size < sizeof(hdr) ? page_size : sizeof(hdr);
	if (read_on(hdr, d_page, take, stream) != FLS_OK) { return FLS_ERR_CUDA; }
	PageInfo pi;
	int      rc = parse_page_header(hdr, take, &pi);
	if (rc == FLS_OK) { rc = finish_page_info(&pi, page_size); }
	if (rc != FLS_OK) { return rc; }
	if (!pi.layout->dict_codes) { return FLS_ERR_UNSUPPORTED; }
	if (pi.vec_c == 0) { return FLS_OK; }
	std::vector<void*> owned;
	const uint8_t*     rvals = nullptr;
	uint64_t           rsize = 0;
	if (pi.layout->ib_rec != kNoBuf) {
		const uint32_t b = pi.layout->ib_rec;
		rc               = decode_rec_on(d_page + pi.off[b], pi.size[b], 4u, &owned, &rvals, &rsize, stream);
	}
	ColDesc c {};
	if (rc == FLS_OK) {
		rc = build_page_column(pi, d_page, 32, nullptr, 0, FLS_TRANSPOSED, reinterpret_cast<uint8_t*>(d_codes), &c,
		                       rvals, rsize);
	}
	if (rc == FLS_OK) {
		DecodeArgs a {};
		a.col0      = c;
		a.n_items   = pi.vec_c;
		a.col_shift = kPageShift;
		if (launch_decode(Family::NUM_PATCH, a, stream) != cudaSuccess) { rc = FLS_ERR_CUDA; }
	}
	if (cudaStreamSynchronize(stream) != cudaSuccess && rc == FLS_OK) { rc = FLS_ERR_CUDA; }
	for (void* p : owned) { cudaFree(p); }
	return rc;
}
} // namespace flsgpu
} // extern "C++"

static int describe_pages(const fls_page_column* cols, uint32_t n_cols, std::vector<ColDesc>* descs,
                          std::vector<uint32_t>* queue, Family* fam_out, cudaStream_t stream,
                          std::vector<void*>* owned, std::vector<uint32_t>* col_desc = nullptr) {
	if (!cols || n_cols == 0 || n_cols > 65535) { return FLS_ERR_ARG; }
	descs->clear();
	descs->reserve(n_cols);
	if (col_desc) { col_desc->assign(n_cols, 0); }
	queue->clear();
	Family fam   = Family::NUM;
	bool   any64 = false;
	for (uint32_t i = 0; i < n_cols; ++i) {
		const fls_page_column& pc = cols[i];
		const int              w  = value_width_of(pc.data_type);
		if (!pc.d_page || !pc.d_out || w == 0 || pc.order > FLS_ORIGINAL) { return FLS_ERR_ARG; }
		if ((reinterpret_cast<uintptr_t>(pc.d_out) & 15u) != 0) { return FLS_ERR_ARG; }
		uint8_t        hdr[8 + 4 * 8];
		const uint64_t take = pc.page_size < sizeof(hdr) ? pc.page_size : sizeof(hdr);
		if (read_on(hdr, pc.d_page, take, stream) != FLS_OK) { return FLS_ERR_CUDA; }
		PageInfo pi;
		int      rc = parse_page_header(hdr, take, &pi);
		if (rc == FLS_OK) { rc = finish_page_info(&pi, pc.page_size); }
		if (rc != FLS_OK) { return rc; }
		const uint8_t* dvals   = nullptr;
		uint32_t       entries = 0;
		if (pi.layout->post == POST_DICT || pi.layout->post == POST_RLE_DICT || pi.layout->dict_codes) {
			if (!pc.d_dict || pc.dict_size < (pc.data_type == DOUBLE ? 8u : 20u)) { return FLS_ERR_FORMAT; }
			uint8_t dh[20];
			if (read_on(dh, pc.d_dict, pc.data_type == DOUBLE ? 8 : 20, stream) != FLS_OK) { return FLS_ERR_CUDA; }
			if (pc.data_type == DOUBLE) {
				// a double dictionary is its entry_c values, raw, after dict_hdr_t (TDic<dbl_pt>::Decompress,
				// src/cor/lyt/dic/dic.cpp:150-153)
				std::memcpy(&entries, dh + 4, 4);
				if (8 + 8ull * entries > pc.dict_size) { return FLS_ERR_FORMAT; }
				dvals = pc.d_dict + 8;
			} else if (dh[8] == 255) {
				uint64_t voff = 0;
				rc            = int_dictionary_values(dh, pc.dict_size, w, &voff, &entries);
				if (rc != FLS_OK) { return rc; }
				dvals = pc.d_dict + voff;
			} else {
				// entries FFOR-packed in rec blocks (dictionaries of 1024 entries and more)
				std::memcpy(&entries, dh + 4, 4);
				uint64_t n = 0;
				rc         = decode_rec_on(pc.d_dict + 8, pc.dict_size - 8, static_cast<uint32_t>(w / 8), owned, &dvals,
				                           &n, stream);
				if (rc != FLS_OK) { return rc; }
				if (n < static_cast<uint64_t>(entries) * (w / 8)) { return FLS_ERR_FORMAT; }
			}
		}
		const uint8_t* rvals = nullptr;
		uint64_t       rsize = 0;
		// the reference has no rec buffers of doubles (THzlDeCmp<double>::decompress_buf aborts,
		// src/cor/eng/hzl_de_cmp.cpp:37-40): RLE _REC pages of a double column are not a format
		if (pc.data_type == DOUBLE && pi.layout->ib_rec != kNoBuf && pi.layout->post == POST_RLE) {
			return FLS_ERR_UNSUPPORTED;
		}
		if (pi.layout->ib_rec != kNoBuf) {
			const uint32_t b = pi.layout->ib_rec;
			rc = decode_rec_on(pc.d_page + pi.off[b], pi.size[b], rec_elem_bytes(pi.layout, w), owned, &rvals, &rsize,
			                   stream);
			if (rc != FLS_OK) { return rc; }
		}
		if (descs->size() + (pi.layout->dict_codes ? 2 : 1) > 65535) { return FLS_ERR_ARG; }
		if (pi.layout->dict_codes) {
			if (entries == 0 || !dvals) { return FLS_ERR_FORMAT; }
			uint8_t* codes = nullptr;
			if (pi.vec_c &&
			    cudaMallocAsync(reinterpret_cast<void**>(&codes), static_cast<uint64_t>(pi.vec_c) * 1024 * 4, stream) !=
			        cudaSuccess) {
				return FLS_ERR_CUDA;
			}
			if (codes) { owned->push_back(codes); }
			ColDesc a {};
			rc = build_page_column(pi, pc.d_page, 32, nullptr, 0, FLS_TRANSPOSED, codes, &a, rvals, rsize);
			if (rc != FLS_OK) { return rc; }
			ColDesc g {};
			g.ws       = 32;
			g.e        = static_cast<uint8_t>(w / 8);
			g.enc      = ENC_RAW;
			g.post     = POST_DICT;
			g.order    = pc.order;
			g.layout   = LAYOUT_ARRAYS;
			g.n_vec    = pi.vec_c;
			g.bw_const = 32;
			g.packed   = codes;
			g.dict     = dvals;
			g.entry_c  = entries;
			g.out      = static_cast<uint8_t*>(pc.d_out);
			const uint32_t ia = static_cast<uint32_t>(descs->size());
			descs->push_back(a);
			descs->push_back(g);
			for (uint32_t v = 0; v < pi.vec_c; ++v) { queue->push_back((ia << kPageShift) | v); }
			for (uint32_t v = 0; v < pi.vec_c; ++v) { queue->push_back(((ia + 1) << kPageShift) | v); }
			if (col_desc) { (*col_desc)[i] = ia + 1; }
			fam = Family::GATHER;
			if (g.e == 8) { any64 = true; }
			continue;
		}
		const uint8_t* r2      = nullptr;
		uint64_t       r2_size = 0;
		if (pi.layout->ib_rec2 != kNoBuf) {
			// REC2: the rsum bases (u16) are a rec buffer too
			const uint32_t b = pi.layout->ib_rec2;
			rc = decode_rec_on(pc.d_page + pi.off[b], pi.size[b], 2u, owned, &r2, &r2_size, stream);
			if (rc != FLS_OK) { return rc; }
		}
		ColDesc d {};
		rc = build_page_column(pi, pc.d_page, w, dvals, entries, pc.order, static_cast<uint8_t*>(pc.d_out), &d, rvals,
		                       rsize, r2, r2_size);
		if (rc != FLS_OK) { return rc; }
		if (post_is_gather(d.post)) { fam = Family::GATHER; }
		if (d.ws == 64) { any64 = true; }
		const uint32_t id = static_cast<uint32_t>(descs->size());
		descs->push_back(d);
		for (uint32_t v = 0; v < pi.vec_c; ++v) { queue->push_back((id << kPageShift) | v); }
		if (col_desc) { (*col_desc)[i] = id; }
	}
	// group the work items by kernel specialisation so that warps run long stretches of one code path (the
	// outputs do not depend on the order)
	// class-major: plain streams, patched streams, gathers (a plan then launches each class's own kernel)
	auto key = [&](uint32_t it) {
		const ColDesc& c = (*descs)[it >> kPageShift];
		const uint32_t klass = post_is_gather(c.post) ? 2u : post_is_patch(c.post) ? 1u : 0u;
		return (klass << 30) | (static_cast<uint32_t>(c.ws) << 23) | (c.e << 16) |
		       (c.enc << 8) | (c.post << 4) | c.order;
	};
	if (descs->size() > 1) {
		std::stable_sort(queue->begin(), queue->end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
	}
	if (fam == Family::GATHER && any64) { fam = Family::ANY; }
	*fam_out = fam;
	return FLS_OK;
}

// One decode of described work items: one launch per item class (plain, patched, gathers) on its own kernel,
// the descriptors and the queue copied in on the stream (a single descriptor needs neither).
static int launch_described(const std::vector<ColDesc>& descs, const std::vector<uint32_t>& queue, cudaStream_t s) {
	if (queue.empty()) { return FLS_OK; }
	DecodeArgs a {};
	a.col_shift = kPageShift;
	Segments sg; // the queue is class-ordered by describe_pages; an unordered one runs on the catch-all kernel
	plan_segments(descs, queue, kPageShift, &sg);
	if (descs.size() == 1 && queue.front() == 0 && queue.back() + 1 == queue.size()) {
		// one descriptor, every vector: the queue is implicit (item v = vector v)
		a.col0    = descs[0];
		a.n_items = queue.size();
		return launch_decode(sg.fam[0], a, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
	}
	ColDesc*  d_cols  = nullptr;
	uint32_t* d_queue = nullptr;
	if (cudaMallocAsync(&d_cols, sizeof(ColDesc) * descs.size(), s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (cudaMallocAsync(&d_queue, sizeof(uint32_t) * queue.size(), s) != cudaSuccess) { return FLS_ERR_CUDA; }
	cudaMemcpyAsync(d_cols, descs.data(), sizeof(ColDesc) * descs.size(), cudaMemcpyHostToDevice, s);
	cudaMemcpyAsync(d_queue, queue.data(), sizeof(uint32_t) * queue.size(), cudaMemcpyHostToDevice, s);
	a.cols = d_cols;
	// copies from pageable host memory are staged before cudaMemcpyAsync returns, so descs/queue may go away
	cudaError_t e = cudaSuccess;
	for (int i = 0; i < sg.n && e == cudaSuccess; ++i) {
		a.queue   = d_queue + sg.begin[i];
		a.n_items = sg.begin[i + 1] - sg.begin[i];
		e         = launch_decode(sg.fam[i], a, s);
	}
	cudaFreeAsync(d_cols, s);
	cudaFreeAsync(d_queue, s);
	return e == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_gpu_decode_pages(const fls_page_column* cols, uint32_t n_cols, fls_stream_t stream) {
	std::vector<ColDesc>  descs;
	std::vector<uint32_t> queue;
	Family                fam = Family::NUM;
	cudaStream_t          s   = static_cast<cudaStream_t>(stream);
	std::vector<void*>    owned;
	struct Free {
		std::vector<void*>& v;
		cudaStream_t        s;
		~Free() {
			for (void* p : v) { cudaFreeAsync(p, s); }
		}
	} free_owned {owned, s};
	int rc = describe_pages(cols, n_cols, &descs, &queue, &fam, s, &owned);
	if (rc != FLS_OK) { return rc; }
	return launch_described(descs, queue, s);
}

// Vectors [first_vec, first_vec + n_vec) of one page (random access by vector, as the reference's
// Reader::get_chunk, src/reader/reader.cpp:19-61, and its declared random_access, include/fastlanes.h:88-106):
// the page's metadata and any whole-page buffer (rec buffers, a patched DICT's code stream) are decoded as for
// the whole page, then only the range's work items run; vector first_vec + i lands at d_out + i * 1024 values.
int fls_gpu_decode_page_vectors(const fls_page_column* col, uint32_t first_vec, uint32_t n_vec, fls_stream_t stream) {
	if (!col) { return FLS_ERR_ARG; }
	std::vector<ColDesc>  descs;
	std::vector<uint32_t> queue, col_desc(1);
	Family                fam = Family::NUM;
	cudaStream_t          s   = static_cast<cudaStream_t>(stream);
	std::vector<void*>    owned;
	struct Free {
		std::vector<void*>& v;
		cudaStream_t        s;
		~Free() {
			for (void* p : v) { cudaFreeAsync(p, s); }
		}
	} free_owned {owned, s};
	int rc = describe_pages(col, 1, &descs, &queue, &fam, s, &owned, &col_desc);
	if (rc != FLS_OK) { return rc; }
	ColDesc&       out = descs[col_desc[0]];
	const uint64_t end = static_cast<uint64_t>(first_vec) + n_vec;
	if (end > out.n_vec) { return FLS_ERR_ARG; }
	// the output descriptor writes vector v at out + v * 1024 * e: shift its base so that first_vec lands at
	// d_out (only addresses of the range are ever formed from it)
	out.out = reinterpret_cast<uint8_t*>(reinterpret_cast<uintptr_t>(out.out) -
	                                     static_cast<uintptr_t>(first_vec) * 1024u * out.e);
	std::vector<uint32_t> part;
	part.reserve(static_cast<size_t>(n_vec) * 2);
	for (const uint32_t it : queue) {
		const uint32_t v = it & ((1u << kPageShift) - 1u);
		if (v >= first_vec && v < end) { part.push_back(it); }
	}
	return launch_described(descs, part, s);
}


int fls_plan_create_filter(const fls_page_column* cols, uint32_t n_cols, const fls_predicate* pred,
                           fls_plan** out_plan) {
	if (!out_plan || !pred || pred->op > FLS_PRED_GE) { return FLS_ERR_ARG; }
	*out_plan = nullptr;
	for (uint32_t i = 0; cols && i < n_cols; ++i) {
		if (cols[i].data_type == DOUBLE) { return FLS_ERR_UNSUPPORTED; }
	}
	std::vector<ColDesc>  descs;
	std::vector<uint32_t> queue;
	Family                fam = Family::NUM;
	std::vector<void*>    owned;
	std::vector<uint32_t> col_desc;
	int                   rc = describe_pages(cols, n_cols, &descs, &queue, &fam, nullptr, &owned, &col_desc);
	if (rc == FLS_OK) {
		// the descriptor that writes each column's output evaluates the predicate (a DICT page's patched code
		// stream, decoded first, still writes its codes)
		for (uint32_t i = 0; i < n_cols; ++i) {
			const uint8_t t = cols[i].data_type;
			descs[col_desc[i]].out_mode =
			    (t == INT8 || t == INT16 || t == INT32 || t == INT64) ? OUT_BITMAP_S : OUT_BITMAP_U;
		}
		rc = make_plan_object(descs, queue, fam, kPageShift, out_plan);
	}
	if (rc == FLS_OK) {
		plan_adopt(*out_plan, std::move(owned));
		Pred p {};
		p.op    = pred->op;
		p.value = static_cast<uint64_t>(pred->value);
		plan_set_filter(*out_plan, p);
	} else {
		cudaDeviceSynchronize();
		for (void* p : owned) { cudaFree(p); }
	}
	return rc;
}

int fls_plan_create_pages(const fls_page_column* cols, uint32_t n_cols, fls_plan** out_plan) {
	if (!out_plan) { return FLS_ERR_ARG; }
	*out_plan = nullptr;
	std::vector<ColDesc>  descs;
	std::vector<uint32_t> queue;
	Family                fam = Family::NUM;
	// headers are read on the legacy default stream: the pages must be in place (e.g. after a device sync)
	std::vector<void*> owned;
	int                rc = describe_pages(cols, n_cols, &descs, &queue, &fam, nullptr, &owned);
	if (rc == FLS_OK) { rc = make_plan_object(descs, queue, fam, kPageShift, out_plan); }
	if (rc == FLS_OK) {
		plan_adopt(*out_plan, std::move(owned)); // decoded rec buffers live as long as the plan
	} else {
		cudaDeviceSynchronize();
		for (void* p : owned) { cudaFree(p); }
	}
	return rc;
}

} // extern "C"
#endif // FLS_HOST_EMULATION
