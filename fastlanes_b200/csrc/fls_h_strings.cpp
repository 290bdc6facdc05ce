// Host side of the string path: page and dictionary metadata, FSST symbol-table import, and the string plan
// (the reference's TColDecoder<str_pt> ExtInitDict + Decompress loop with the materialisation of
// include/fls/encoder/assert_eq.hpp:166-210 and :257-400).
#include "fastlanes.h"
#include "fls_b200.h"
#include "fls_page.h"
#include "fls_runtime.h"
#include "fls_strplan.h"

#include <algorithm>
#include <cstring>
#include <cuda_runtime.h>
#include <memory>
#include <vector>

namespace flsgpu {

// FSST_MAXHEADER (include/fls/cor/prm/fsst/fsst.h:112-114): the dictionary page reserves this many bytes for
// the exported symbol table whatever its length (src/cor/lyt/dic/dic.cpp:99-101).
constexpr uint64_t kFsstMaxHeader = 8 + 1 + 8 + 2048 + 1;

// fsst_import (src/cor/prm/fsst/libfsst.cpp:617-657): 8-byte version word (upper 32 bits 20190218), byte 8 the
// zero-terminated flag, bytes 9..16 the symbol count per length, then the symbol bytes grouped by length in the
// order 2,3,4,5,6,7,8,1; codes are numbered from the flag upward; unused codes decode to "corrupt" (8 bytes).
int fsst_import_table(const uint8_t* buf, uint64_t avail, FsstTable* t, uint64_t* used) {
	if (avail < 17) { return FLS_ERR_FORMAT; }
	uint64_t version = 0;
	std::memcpy(&version, buf, 8);
	if ((version >> 32) != 20190218ull) { return FLS_ERR_FORMAT; }
	const uint32_t zt = buf[8] & 1u;
	uint8_t        hist[8];
	std::memcpy(hist, buf + 9, 8);
	std::memset(t, 0, sizeof(*t));
	t->len[0]     = 1;
	t->sym[0]     = 0;
	uint32_t code = zt;
	uint64_t pos  = 17;
	if (zt) { hist[0] = static_cast<uint8_t>(hist[0] - 1); }
	for (uint32_t l = 1; l <= 8; ++l) {
		for (uint32_t i = 0; i < hist[l & 7]; ++i, ++code) {
			if (code >= 255) { return FLS_ERR_FORMAT; }
			t->len[code] = static_cast<uint8_t>((l & 7) + 1);
			t->sym[code] = 0;
			for (uint32_t j = 0; j < t->len[code]; ++j) {
				if (pos >= avail) { return FLS_ERR_FORMAT; }
				t->sym[code] |= static_cast<uint64_t>(buf[pos++]) << (8 * j);
			}
		}
	}
	while (code < 255) {
		t->sym[code] = 32774747032022883ull; // "corrupt"
		t->len[code] = 8;
		++code;
	}
	if (used) { *used = pos; }
	return FLS_OK;
}

// fsst12_import (src/cor/prm/fsst12/libfsst12.cpp:363-389): 8-byte version word (upper 32 bits 20190218),
// lenHisto (8 u16 symbol counts) at byte 8, from byte 24 every symbol as its length byte and that many
// little-endian bytes; codes past the symbol count decode as the 8 bytes "corrupt".  Symbol lengths above 8 and
// more than 4096 symbols (which the reference would write past its table for) are format errors.
int fsst12_import_table(const uint8_t* buf, uint64_t avail, Fsst12Table* t, uint64_t* used) {
	if (avail < 24) { return FLS_ERR_FORMAT; }
	uint64_t version = 0;
	std::memcpy(&version, buf, 8);
	if ((version >> 32) != 20190218ull) { return FLS_ERR_FORMAT; }
	uint16_t hist[8];
	std::memcpy(hist, buf + 8, 16);
	uint32_t count = 0;
	for (const uint16_t h : hist) { count += h; }
	if (count > 4096) { return FLS_ERR_FORMAT; }
	std::memset(t, 0, sizeof(*t));
	uint64_t pos = 24;
	for (uint32_t code = 0; code < count; ++code) {
		if (pos >= avail) { return FLS_ERR_FORMAT; }
		const uint32_t l = buf[pos++];
		if (l > 8 || pos + l > avail) { return FLS_ERR_FORMAT; }
		t->len[code] = static_cast<uint8_t>(l);
		for (uint32_t j = 0; j < l; ++j) { t->sym[code] |= static_cast<uint64_t>(buf[pos++]) << (8 * j); }
	}
	for (uint32_t code = count; code < 4096; ++code) {
		t->sym[code] = 32774747032022883ull; // "corrupt"
		t->len[code] = 8;
	}
	if (used) { *used = pos; }
	return FLS_OK;
}

namespace {

// Row-stream layouts of the string expressions (roles as in the integer table of fls_h_page.cpp; ib_vals of a
// DICT_RLE page holds the u32 code runs).  kind: STR_*.
// patched: the DICT page's codes are a patched FFOR / DELTA stream, decoded once at plan creation
// (decode_patched_codes) and then read as an UNCOMPRESSED code stream.
struct StrLayout {
	uint8_t exp_t, var, arr_c, ws, enc, post, ib_bw, ib_base, ib_packed, ib_lane, ib_vals, kind;
	uint8_t patched = 0;
};
const StrLayout* str_layout(uint8_t exp_t, uint8_t var) {
	// DICT_FRQ (exp_t 9) pages are DICT pages over a frequency-ordered dictionary (dict_exp.hpp:208)
	exp_t = exp_t == 9 ? 8 : exp_t;
	static const StrLayout t[] = {
	    {8, 1, 1, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT},   // DICT UNCOMPRESSED
	    {8, 2, 3, 32, ENC_FFOR, POST_NONE, 0, 1, 2, kNoBuf, kNoBuf, STR_DICT},            // DICT FFOR_NO_PATCH
	    {8, 7, 4, 32, ENC_DELTA, POST_NONE, 1, 2, 3, 0, kNoBuf, STR_DICT},                // DICT DELTA_NO_PATCH
	    {8, 3, 5, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT FFOR_LL_PATCH
	    {8, 4, 5, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT FFOR_S_PATCH
	    {8, 5, 5, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT FFOR_B_PATCH
	    {8, 6, 5, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT FFOR_S_PATCH_REC
	    {8, 8, 6, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT DELTA_LL_PATCH
	    {8, 9, 6, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT DELTA_S_PATCH
	    {8, 10, 6, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // DICT DELTA_B_PATCH
	    {8, 11, 6, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 0, kNoBuf, kNoBuf, STR_DICT, 1}, // ..._B_PATCH_REC
	    {11, 1, 2, 16, ENC_RAW, POST_RLE, kNoBuf, kNoBuf, 1, kNoBuf, 0, STR_DICT},        // DICT_RLE UNCOMPRESSED
	    {11, 2, 5, 16, ENC_DELTA, POST_RLE, 2, 3, 4, 1, 0, STR_DICT},                     // DICT_RLE DELTA_NO_PATCH
	    {7, 1, 2, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 1, kNoBuf, kNoBuf, STR_FSST},   // FSST
	    {7, 2, 5, 32, ENC_DELTA, POST_NONE, 2, 3, 4, 1, kNoBuf, STR_FSST},                // FSST DELTA_NO_PATCH
	    {20, 1, 2, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 1, kNoBuf, kNoBuf, STR_FSST12}, // FSST12
	    {20, 2, 5, 32, ENC_DELTA, POST_NONE, 2, 3, 4, 1, kNoBuf, STR_FSST12},              // FSST12 DELTA_NO_PATCH
	    {3, 1, 2, 32, ENC_RAW, POST_NONE, kNoBuf, kNoBuf, 1, kNoBuf, kNoBuf, STR_BYTES},  // BYTE_ARR
	    {3, 2, 5, 32, ENC_DELTA, POST_NONE, 2, 3, 4, 1, kNoBuf, STR_BYTES},               // BYTE_ARR DELTA_NO_PATCH
	};
	for (const auto& e : t) {
		if (e.exp_t == exp_t && e.var == var) { return &e; }
	}
	return nullptr;
}

template <class T>
struct DevArr {
	T* p = nullptr;
	~DevArr() {
		if (p) { cudaFree(p); }
	}
	bool alloc(size_t n) { return cudaMalloc(&p, (n ? n : 1) * sizeof(T)) == cudaSuccess; }
};

} // namespace
} // namespace flsgpu

using namespace flsgpu;

struct fls_string_plan {
	StrArgs                  args {};
	DevArr<FsstTable>        table;
	DevArr<Fsst12Table>      table12;
	DevArr<uint32_t>         dict_ends;
	DevArr<uint32_t>         dict_rows; // packed start | length << 24 of every entry, when they fit
	DevArr<uint8_t>          dict_bytes;
	DevArr<uint64_t>         vec_total;
	DevArr<uint64_t>         vec_base;
	DevArr<uint32_t>         codes; // patched DICT pages: their decoded code stream
	DevArr<uint32_t>         row_len; // FSST12 pages: every row's decoded length
	uint32_t                 dyn_smem = 0;
	int                      warps    = 0; // warps per CTA of the materialising kernel
	uint64_t                 n_rows   = 0;
	// single-pass DICT decode (k_dict_pass): DICT pages whose dictionary has a packed row table
	bool                     single   = false;
	DevArr<StrArgs>          dargs;    // the plan's arguments in device memory (item_base 0)
	DevArr<uint64_t>         lb;       // ticket + one look-back word per vector, zeroed before every decode
	int                      sp_warps = 0;
	uint32_t                 sp_smem  = 0, sp_dict_cap = 0, sp_tab_cap = 0;
	// single-pass FSST / BYTE_ARR decode (k_stream_single), look-back words in lb
	bool                     stream_single = false;
	// a measure() whose per-vector totals and bases the next decode() takes over (the usual measure, allocate,
	// decode sequence runs the lengths pass once)
	mutable bool             measured = false;
};

extern "C" {

int fls_string_plan_create(const uint8_t* d_page, uint64_t page_size, const uint8_t* d_dict, uint64_t dict_size,
                           fls_string_plan** out) {
	if (!out || !d_page) { return FLS_ERR_ARG; }
	*out = nullptr;
	Device* dev = current_device();
	if (!dev) { return FLS_ERR_CUDA; }
	uint8_t hdr[8 + 4 * 6];
	const uint64_t take = page_size < sizeof(hdr) ? page_size : sizeof(hdr);
	if (take < 8 || cudaMemcpy(hdr, d_page, take, cudaMemcpyDeviceToHost) != cudaSuccess) { return FLS_ERR_FORMAT; }
	const StrLayout* L = str_layout(hdr[0], hdr[1]);
	if (!L) { return FLS_ERR_UNSUPPORTED; }
	PageInfo pi {};
	pi.exp_t = hdr[0];
	pi.var   = hdr[1];
	std::memcpy(&pi.vec_c, hdr + 4, 2);
	pi.arr_c = L->arr_c;
	if (take < 8ull + 4 * pi.arr_c) { return FLS_ERR_FORMAT; }
	for (uint32_t i = 0; i < pi.arr_c; ++i) { std::memcpy(&pi.off[i], hdr + 8 + 4 * i, 4); }
	pi.ep_off  = 8 + 4 * pi.arr_c;
	pi.meta_sz = pi.ep_off + 4ull * pi.arr_c * (pi.vec_c ? pi.vec_c - 1 : 0);
	int rc     = finish_page_info(&pi, page_size);
	if (rc != FLS_OK) { return rc; }
	std::unique_ptr<fls_string_plan> p(new fls_string_plan());
	StrArgs&                         a = p->args;
	ColDesc&                         c = a.col;
	c        = ColDesc {};
	c.ws     = L->ws;
	c.e      = 4;
	c.enc    = L->enc;
	c.post   = L->post;
	c.order  = 1;
	c.layout = LAYOUT_PAGE;
	c.arr_c  = static_cast<uint8_t>(pi.arr_c);
	c.n_vec  = pi.vec_c;
	c.ib_bw = L->ib_bw, c.ib_base = L->ib_base, c.ib_packed = L->ib_packed, c.ib_lane_bases = L->ib_lane;
	c.ib_vals = L->ib_vals;
	for (uint32_t i = 0; i < pi.arr_c; ++i) {
		c.buf[i]      = d_page + pi.off[i];
		c.buf_size[i] = pi.size[i];
	}
	c.ep      = reinterpret_cast<const uint32_t*>(d_page + pi.ep_off);
	if (L->patched) {
		// decoded once here; the string kernels then read a raw 32-bit code stream
		if (!p->codes.alloc(static_cast<size_t>(pi.vec_c) * 1024)) { return FLS_ERR_CUDA; }
		rc = decode_patched_codes(d_page, page_size, p->codes.p, nullptr);
		if (rc != FLS_OK) { return rc; }
		c          = ColDesc {};
		c.ws       = 32;
		c.e        = 4;
		c.enc      = ENC_RAW;
		c.post     = POST_NONE;
		c.order    = 1;
		c.layout   = LAYOUT_ARRAYS;
		c.n_vec    = pi.vec_c;
		c.bw_const = 32;
		c.packed   = reinterpret_cast<const uint8_t*>(p->codes.p);
	}
	a.kind    = L->kind;
	a.status  = dev->status;
	p->n_rows = static_cast<uint64_t>(pi.vec_c) * 1024;
	if (!p->vec_total.alloc(pi.vec_c + 1) || !p->vec_base.alloc(pi.vec_c + 1)) { return FLS_ERR_CUDA; }
	a.vec_total = p->vec_total.p;
	a.vec_base  = p->vec_base.p;
	if (L->kind == STR_FSST12) {
		if (!p->row_len.alloc(static_cast<size_t>(pi.vec_c) * 1024)) { return FLS_ERR_CUDA; }
		a.row_len = p->row_len.p;
	}
	if (!p->table.alloc(1)) { return FLS_ERR_CUDA; }
	FsstTable tab {};
	if (L->kind == STR_FSST12) {
		// dict_hdr | exported FSST12 table (at most FSST12_MAXHEADER = 36888 bytes)
		if (!d_dict || dict_size < 8 + 24) { return FLS_ERR_FORMAT; }
		const uint64_t       head = dict_size < 8 + 36888 ? dict_size : 8 + 36888;
		std::vector<uint8_t> h(head);
		if (cudaMemcpy(h.data(), d_dict, head, cudaMemcpyDeviceToHost) != cudaSuccess) { return FLS_ERR_CUDA; }
		std::unique_ptr<Fsst12Table> t12(new Fsst12Table());
		rc = fsst12_import_table(h.data() + 8, head - 8, t12.get(), nullptr);
		if (rc != FLS_OK) { return rc; }
		if (!p->table12.alloc(1) ||
		    cudaMemcpy(p->table12.p, t12.get(), sizeof(Fsst12Table), cudaMemcpyHostToDevice) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		a.table12 = p->table12.p;
	} else if (L->kind != STR_BYTES) {
		// DICT: dict_hdr | FSST table slot | entry_c u32 lengths | bytes.  FSST column: dict_hdr | exported table.
		if (!d_dict || dict_size < 8 + 17) { return FLS_ERR_FORMAT; }
		const uint64_t head = L->kind == STR_DICT ? 8 + kFsstMaxHeader : dict_size;
		if (head > dict_size) { return FLS_ERR_FORMAT; }
		std::vector<uint8_t> h(head);
		if (cudaMemcpy(h.data(), d_dict, head, cudaMemcpyDeviceToHost) != cudaSuccess) { return FLS_ERR_CUDA; }
		rc = fsst_import_table(h.data() + 8, head - 8, &tab, nullptr);
		if (rc != FLS_OK) { return rc; }
		if (L->kind == STR_DICT) {
			uint32_t entry_c = 0;
			std::memcpy(&entry_c, h.data() + 4, 4);
			const uint64_t lens_off = 8 + kFsstMaxHeader;
			const uint64_t comp_off = lens_off + 4ull * entry_c;
			if (entry_c == 0 || comp_off > dict_size) { return FLS_ERR_FORMAT; }
			const uint64_t comp_size = dict_size - comp_off;
			const uint64_t cap       = comp_size * 8 + 16;
			if (!p->dict_ends.alloc(entry_c) || !p->dict_bytes.alloc(cap)) { return FLS_ERR_CUDA; }
			cudaMemcpy(p->table.p, &tab, sizeof(tab), cudaMemcpyHostToDevice);
			if (launch_fsst_dict(d_dict + lens_off, d_dict + comp_off, comp_size, entry_c, p->table.p,
			                     p->dict_ends.p, p->dict_bytes.p, cap, dev->status, nullptr) != cudaSuccess) {
				return FLS_ERR_CUDA;
			}
			uint32_t last = 0;
			if (cudaMemcpy(&last, p->dict_ends.p + entry_c - 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
				return FLS_ERR_CUDA;
			}
			if (last < (1u << 24)) {
				// the row table of the materialising pass: start | length << 24 when every entry is < 256 bytes
				std::vector<uint32_t> ends(entry_c);
				if (cudaMemcpy(ends.data(), p->dict_ends.p, 4ull * entry_c, cudaMemcpyDeviceToHost) != cudaSuccess) {
					return FLS_ERR_CUDA;
				}
				bool     fits  = true;
				uint32_t start = 0;
				for (uint32_t c = 0; c < entry_c && fits; ++c) {
					fits    = ends[c] >= start && ends[c] - start < 256;
					ends[c] = start | ((ends[c] - start) << 24);
					start   = static_cast<uint32_t>(ends[c] & 0xFFFFFFu) + (ends[c] >> 24);
				}
				if (fits) {
					if (!p->dict_rows.alloc(entry_c) ||
					    cudaMemcpy(p->dict_rows.p, ends.data(), 4ull * entry_c, cudaMemcpyHostToDevice) != cudaSuccess) {
						return FLS_ERR_CUDA;
					}
					a.dict_rows = p->dict_rows.p;
				}
			}
			a.entry_c      = entry_c;
			a.dict_ends    = p->dict_ends.p;
			a.dict_bytes   = p->dict_bytes.p;
			a.dict_bytes_n = last;
		}
	}
	if (cudaMemcpy(p->table.p, &tab, sizeof(tab), cudaMemcpyHostToDevice) != cudaSuccess) { return FLS_ERR_CUDA; }
	a.table = p->table.p;
	// shared memory of the string kernels: the lengths pass keeps the dictionary end offsets there (up to 64 KB
	// of them) after its per-warp areas; the materialising pass the decoded dictionary bytes (its end offsets are
	// looked up a batch ahead from global memory) when at least 8 warps still fit beside them
	// 16-bit code rows: fewer than 65535 entries and at most 2 KB of packed codes per vector (16-bit lanes, or
	// bit widths up to 16 in every vector)
	a.rows16 = a.kind == STR_DICT && a.entry_c < 0xFFFFu && (c.ws == 16 || c.enc != ENC_RAW);
	if (a.rows16 && c.ws == 32) {
		std::vector<uint8_t> bw(c.buf_size[c.ib_bw]);
		if (!bw.empty() && cudaMemcpy(bw.data(), c.buf[c.ib_bw], bw.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		for (const uint8_t w : bw) { a.rows16 = a.rows16 && w <= 16; }
	}
	const uint32_t per_warp = str_smem_per_warp(a.rows16);
	const uint64_t budget   = 224 * 1024 - (a.kind == STR_FSST12 ? kStrFsst12Smem : 0u);
	const uint64_t dict_sm  = (a.dict_bytes_n + 15) & ~15ull;
	a.ends_in_smem          = a.kind == STR_DICT && str_ends_smem(a) <= kStrEndsSmemMax;
	a.dict_in_smem          = false;
	uint64_t w              = budget / per_warp;
	if (a.kind == STR_DICT && dict_sm < budget && (budget - dict_sm) / per_warp >= 8) {
		a.dict_in_smem = true;
		w              = (budget - dict_sm) / per_warp;
	}
	p->warps    = static_cast<int>(w < kStrMaxWarps ? w : kStrMaxWarps);
	p->dyn_smem = static_cast<uint32_t>(p->warps * per_warp + (a.dict_in_smem ? dict_sm : 0u));
	if (a.kind == STR_DICT && a.dict_rows && pi.vec_c > 0) {
		// single-pass decode: the dictionary and its row table in shared memory when at least 8 warps still fit
		p->single            = true;
		const uint32_t   pw  = dict_pass_smem_per_warp(a.rows16);
		const uint64_t   tab = (4ull * a.entry_c + 15) & ~15ull;
		const uint64_t   all = 224 * 1024;
		uint64_t         sw  = all / pw;
		if (dict_sm + tab < all && (all - dict_sm - tab) / pw >= 8) {
			p->sp_dict_cap = static_cast<uint32_t>(dict_sm);
			p->sp_tab_cap  = a.entry_c;
			sw             = (all - dict_sm - tab) / pw;
		}
		p->sp_warps = static_cast<int>(sw < kStrMaxWarps ? sw : kStrMaxWarps);
		p->sp_smem  = static_cast<uint32_t>(p->sp_warps * pw + (p->sp_dict_cap ? dict_sm + tab : 0u));
		if (!p->dargs.alloc(1) || !p->lb.alloc(1ull + pi.vec_c) ||
		    cudaMemcpy(p->dargs.p, &a, sizeof(StrArgs), cudaMemcpyHostToDevice) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
	}
	if ((a.kind == STR_FSST || a.kind == STR_BYTES) && pi.vec_c > 0) {
		p->stream_single = true;
		if (!p->lb.alloc(1ull + pi.vec_c)) { return FLS_ERR_CUDA; }
	}
	*out                    = p.release();
	return FLS_OK;
}

int fls_string_plan_rows(const fls_string_plan* p, uint64_t* n_rows) {
	if (!p || !n_rows) { return FLS_ERR_ARG; }
	*n_rows = p->n_rows;
	return FLS_OK;
}

static int run_totals(const fls_string_plan* p, cudaStream_t s) {
	if (p->args.col.n_vec == 0) { return FLS_OK; }
	if (launch_str_lengths(p->args, 0, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (launch_scan_totals(p->vec_total.p, p->vec_base.p, p->args.col.n_vec, s) != cudaSuccess) { return FLS_ERR_CUDA; }
	return FLS_OK;
}

int fls_string_plan_measure(fls_string_plan* p, uint64_t* n_bytes, fls_stream_t stream) {
	if (!p || !n_bytes) { return FLS_ERR_ARG; }
	cudaStream_t s  = static_cast<cudaStream_t>(stream);
	p->measured     = false;
	const int    rc = run_totals(p, s);
	if (rc != FLS_OK) { return rc; }
	*n_bytes = 0;
	if (p->args.col.n_vec == 0) { return FLS_OK; }
	if (cudaMemcpyAsync(n_bytes, p->vec_base.p + p->args.col.n_vec, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	if (cudaStreamSynchronize(s) != cudaSuccess) { return FLS_ERR_CUDA; }
	p->measured = true;
	return FLS_OK;
}

// The single-pass DICT decode of one plan: one memset of its look-back words and one launch.
static int single_pass_decode(const fls_string_plan* p, uint32_t* d_offsets, uint8_t* d_bytes, uint64_t cap,
                              cudaStream_t s) {
	const uint32_t n_vec = p->args.col.n_vec;
	if (cudaMemsetAsync(p->lb.p, 0, 8ull * (1 + n_vec), s) != cudaSuccess) { return FLS_ERR_CUDA; }
	StrSetArgs x {};
	x.cols        = p->dargs.p;
	x.chunk_w     = static_cast<uint32_t>(p->sp_warps);
	x.n_chunks    = (n_vec + x.chunk_w - 1) / x.chunk_w;
	x.flags       = p->lb.p;
	x.status      = p->args.status;
	x.out_offsets = d_offsets;
	x.out_bytes   = d_bytes;
	x.out_cap     = cap;
	x.dict_cap    = p->sp_dict_cap;
	x.tab_cap     = p->sp_tab_cap;
	return launch_dict_pass(x, p->args.rows16, p->sp_warps, p->sp_smem, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_string_plan_decode(const fls_string_plan* p, uint32_t* d_offsets, uint8_t* d_bytes, uint64_t bytes_cap,
                           fls_stream_t stream) {
	if (!p || !d_offsets || (!d_bytes && bytes_cap)) { return FLS_ERR_ARG; }
	if ((reinterpret_cast<uintptr_t>(d_bytes) & 15u) != 0 || bytes_cap >= (1ull << 32)) { return FLS_ERR_ARG; }
	cudaStream_t s  = static_cast<cudaStream_t>(stream);
	if (p->single) {
		p->measured = false;
		return single_pass_decode(p, d_offsets, d_bytes, bytes_cap, s);
	}
	if (p->stream_single) {
		// one memset of the look-back words and one launch
		p->measured = false;
		StrArgs a   = p->args;
		a.offsets   = d_offsets;
		a.bytes     = d_bytes;
		a.bytes_cap = bytes_cap;
		if (cudaMemsetAsync(p->lb.p, 0, 8ull * (1 + a.col.n_vec), s) != cudaSuccess) { return FLS_ERR_CUDA; }
		return launch_stream_single(a, p->lb.p, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
	}
	// the totals of a measure() just before (complete: measure synchronised its stream) are still valid; a
	// decode captured into a graph always computes its own (each replay must)
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) { return FLS_ERR_CUDA; }
	int rc      = p->measured && cs == cudaStreamCaptureStatusNone ? FLS_OK : run_totals(p, s);
	p->measured = false;
	if (rc != FLS_OK) { return rc; }
	if (p->args.col.n_vec == 0) {
		return cudaMemsetAsync(d_offsets, 0, 4, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
	}
	StrArgs a   = p->args;
	a.offsets   = d_offsets;
	a.bytes     = d_bytes;
	a.bytes_cap = bytes_cap;
	return launch_str_materialize(a, p->warps, p->dyn_smem, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}



int fls_string_plan_destroy(fls_string_plan* p) {
	delete p;
	return FLS_OK;
}

} // extern "C"

// A set of single-pass DICT string plans decoded by one launch (k_dict_pass over every column's vectors).
struct fls_string_set {
	std::vector<StrArgs> args;     // every column's arguments: item_base, and the outputs once bound
	DevArr<StrArgs>      cols;     // the same in device memory
	DevArr<uint32_t>     chunk_col, chunk_v0;
	DevArr<uint64_t>     lb;       // ticket + one look-back word per vector of every column
	uint64_t             n_items  = 0;
	uint32_t             n_chunks = 0;
	int                  warps    = 0;
	uint32_t             smem = 0, dict_cap = 0, tab_cap = 0;
	bool                 rows16 = true, bound = false;
	int*                 status = nullptr;
};

extern "C" {

int fls_string_set_create(const fls_string_plan* const* plans, uint32_t n, fls_string_set** out) {
	if (!out || !plans || n == 0) { return FLS_ERR_ARG; }
	*out = nullptr;
	std::unique_ptr<fls_string_set> set(new fls_string_set());
	uint64_t dict_max = 0, tab_max = 0;
	for (uint32_t i = 0; i < n; ++i) {
		if (!plans[i]) { return FLS_ERR_ARG; }
		if (!plans[i]->single) { return FLS_ERR_UNSUPPORTED; } // DICT pages with a packed row table only
		StrArgs a   = plans[i]->args;
		a.item_base = set->n_items;
		set->args.push_back(a);
		set->n_items += a.col.n_vec;
		set->rows16 = set->rows16 && a.rows16;
		dict_max    = std::max<uint64_t>(dict_max, (a.dict_bytes_n + 15) & ~15ull);
		tab_max     = std::max<uint64_t>(tab_max, a.entry_c);
		set->status = a.status;
	}
	const uint32_t pw  = dict_pass_smem_per_warp(set->rows16);
	const uint64_t tab = (4 * tab_max + 15) & ~15ull;
	const uint64_t all = 224 * 1024;
	uint64_t       w   = all / pw;
	if (dict_max + tab < all && (all - dict_max - tab) / pw >= 8) {
		set->dict_cap = static_cast<uint32_t>(dict_max);
		set->tab_cap  = static_cast<uint32_t>(tab_max);
		w             = (all - dict_max - tab) / pw;
	}
	set->warps = static_cast<int>(w < kStrMaxWarps ? w : kStrMaxWarps);
	set->smem  = static_cast<uint32_t>(set->warps * pw + (set->dict_cap ? dict_max + tab : 0u));
	// chunks of `warps` vectors that never cross a column, in column order
	std::vector<uint32_t> cc, cv;
	for (uint32_t i = 0; i < n; ++i) {
		for (uint32_t v = 0; v < set->args[i].col.n_vec; v += static_cast<uint32_t>(set->warps)) {
			cc.push_back(i);
			cv.push_back(v);
		}
	}
	set->n_chunks = static_cast<uint32_t>(cc.size());
	if (!set->cols.alloc(n) || !set->lb.alloc(1 + set->n_items) || !set->chunk_col.alloc(cc.size()) ||
	    !set->chunk_v0.alloc(cv.size())) {
		return FLS_ERR_CUDA;
	}
	if (!cc.empty() && (cudaMemcpy(set->chunk_col.p, cc.data(), 4 * cc.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
	                    cudaMemcpy(set->chunk_v0.p, cv.data(), 4 * cv.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
		return FLS_ERR_CUDA;
	}
	*out = set.release();
	return FLS_OK;
}

int fls_string_set_bind(fls_string_set* set, uint32_t* const* d_offsets, uint8_t* const* d_bytes,
                        const uint64_t* bytes_caps) {
	if (!set || !d_offsets || !d_bytes || !bytes_caps) { return FLS_ERR_ARG; }
	for (size_t i = 0; i < set->args.size(); ++i) {
		if (!d_offsets[i] || (!d_bytes[i] && bytes_caps[i]) || (reinterpret_cast<uintptr_t>(d_bytes[i]) & 15u) != 0 ||
		    bytes_caps[i] >= (1ull << 32)) {
			return FLS_ERR_ARG;
		}
		set->args[i].offsets   = d_offsets[i];
		set->args[i].bytes     = d_bytes[i];
		set->args[i].bytes_cap = bytes_caps[i];
	}
	if (cudaMemcpy(set->cols.p, set->args.data(), sizeof(StrArgs) * set->args.size(), cudaMemcpyHostToDevice) !=
	    cudaSuccess) {
		return FLS_ERR_CUDA;
	}
	set->bound = true;
	return FLS_OK;
}

int fls_string_set_decode(const fls_string_set* set, fls_stream_t stream) {
	if (!set || !set->bound) { return FLS_ERR_ARG; }
	cudaStream_t s = static_cast<cudaStream_t>(stream);
	if (cudaMemsetAsync(set->lb.p, 0, 8ull * (1 + set->n_items), s) != cudaSuccess) { return FLS_ERR_CUDA; }
	StrSetArgs x {};
	x.cols      = set->cols.p;
	x.chunk_col = set->chunk_col.p;
	x.chunk_v0  = set->chunk_v0.p;
	x.n_chunks  = set->n_chunks;
	x.chunk_w   = static_cast<uint32_t>(set->warps);
	x.flags     = set->lb.p;
	x.status    = set->status;
	x.dict_cap  = set->dict_cap;
	x.tab_cap   = set->tab_cap;
	return launch_dict_pass(x, set->rows16, set->warps, set->smem, s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

int fls_string_set_destroy(fls_string_set* set) {
	delete set;
	return FLS_OK;
}

} // extern "C"
