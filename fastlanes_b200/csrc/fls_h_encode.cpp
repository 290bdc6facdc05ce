// Encoder side used for workloads, round trips and trial encodes: RLE pages, FSST symbol tables and
// string-dictionary pages.  Decoding never depends on these encoders being the reference's own: every page they
// write follows the reference's byte format, checked by the tests against the reference's encoder output.
//
//   RLE DELTA_NO_PATCH (int64 expression 6; include/fls/cor/exp/rle/rle_exp.hpp:56-74): per vector the run
//   values (T) and a u16 run index in original order (src/cor/lyt/vec.cpp:50-71), the index transposed, its
//   first row kept as lane bases, delta-encoded and FFOR bit-packed (src/cor/prm/rle/rle_compress.cpp:10-45,
//   src/cor/prm/rsum/rsum_compress.cpp:10-22, src/cor/prm/ffor/ffor_compress.cpp:10-26).
//   FSST: a symbol table of at most 255 symbols of 1..8 bytes, built by the iterative counting procedure of
//   FSST (Boncz, Neumann, Leis: "FSST: Fast Random Access String Compression", VLDB 2020): parse a sample
//   with the current table, count symbols and adjacent symbol pairs, keep the 255 candidates of highest gain
//   (count x length), repeat.  Strings are compressed greedily by longest match, escape 255 for other bytes.
//   The table is serialised in fsst_export's format (read back by fsst_import,
//   src/cor/prm/fsst/libfsst.cpp:617-657).
//   String DICT FFOR_NO_PATCH (str expression 3): dictionary page = dict_hdr_t | FSST table (FSST_MAXHEADER
//   slot) | entry_c u32 compressed lengths | compressed bytes (src/cor/lyt/dic/dic.cpp:88-111); the codes are a
//   u32 FFOR page with the DICT header (include/fls/cor/exp/dict/dict_exp.hpp:51-60).  Unlike the reference's
//   TDic::serialize, the lengths stored are the true compressed lengths of each entry.
#include "fastlanes.h"
#include "fls_b200.h"
#include "fls_page.h"
#include "fls_runtime.h"

#include <algorithm>
#include <cstring>
#include <cuda_runtime.h>
#include <unordered_map>
#include <vector>

namespace flsgpu {
namespace {

// ------------------------------------------------------------------------------------------------------------
// FSST table construction
// ------------------------------------------------------------------------------------------------------------
struct Sym {
	uint64_t val;
	uint32_t len;
};

inline uint64_t load_bytes(const uint8_t* p, uint32_t n) {
	uint64_t v = 0;
	std::memcpy(&v, p, n);
	return v;
}

struct SymTable {
	std::vector<Sym>                          syms;  // code order
	std::unordered_map<uint64_t, uint32_t>    by_len[9];

	void index() {
		for (auto& m : by_len) { m.clear(); }
		for (uint32_t c = 0; c < syms.size(); ++c) { by_len[syms[c].len][syms[c].val] = c; }
	}
	// longest symbol matching at s[0..n): returns code, or -1
	int match(const uint8_t* s, uint32_t n, uint32_t* mlen) const {
		for (uint32_t L = n < 8 ? n : 8; L >= 1; --L) {
			auto it = by_len[L].find(load_bytes(s, L));
			if (it != by_len[L].end()) {
				*mlen = L;
				return static_cast<int>(it->second);
			}
		}
		return -1;
	}
};

struct SymKey {
	uint64_t val;
	uint32_t len;
	bool     operator==(const SymKey& o) const { return val == o.val && len == o.len; }
};
struct SymKeyHash {
	size_t operator()(const SymKey& k) const { return std::hash<uint64_t>()(k.val * 0x9E3779B97F4A7C15ull ^ k.len); }
};

SymTable build_table(const std::vector<std::pair<const uint8_t*, uint32_t>>& sample) {
	SymTable t;
	for (int round = 0; round < 5; ++round) {
		// parse the sample with the current table; literal bytes count as 1-byte candidates
		std::unordered_map<SymKey, uint64_t, SymKeyHash> gain;
		for (const auto& [s, n] : sample) {
			uint32_t p = 0;
			SymKey   prev {0, 0};
			while (p < n) {
				uint32_t  len  = 1;
				const int code = t.match(s + p, n - p, &len);
				SymKey    cur {code >= 0 ? t.syms[code].val : s[p], code >= 0 ? len : 1u};
				gain[cur] += cur.len;
				if (prev.len && prev.len + cur.len <= 8) {
					const SymKey pair {prev.val | (cur.val << (8 * prev.len)), prev.len + cur.len};
					gain[pair] += pair.len;
				}
				prev = cur;
				p += cur.len;
			}
		}
		std::vector<std::pair<uint64_t, SymKey>> ranked;
		ranked.reserve(gain.size());
		for (const auto& kv : gain) { ranked.emplace_back(kv.second, kv.first); }
		std::sort(ranked.begin(), ranked.end(), [](const auto& a, const auto& b) {
			if (a.first != b.first) { return a.first > b.first; }
			if (a.second.len != b.second.len) { return a.second.len > b.second.len; }
			return a.second.val < b.second.val;
		});
		t.syms.clear();
		for (const auto& c : ranked) {
			if (t.syms.size() == 255) { break; }
			t.syms.push_back(Sym {c.second.val, c.second.len});
		}
		t.index();
	}
	// code order of fsst_import: lengths 2,3,...,8 first, then 1
	std::stable_sort(t.syms.begin(), t.syms.end(), [](const Sym& a, const Sym& b) {
		const uint32_t ka = a.len == 1 ? 9 : a.len, kb = b.len == 1 ? 9 : b.len;
		return ka < kb;
	});
	t.index();
	return t;
}

uint32_t export_table(const SymTable& t, uint8_t* buf) {
	const uint64_t n       = t.syms.size();
	const uint64_t version = (20190218ull << 32) | (n << 8) | 1ull;
	std::memcpy(buf, &version, 8);
	buf[8] = 0; // not zero-terminated
	uint8_t hist[8] = {};
	for (const auto& s : t.syms) { hist[s.len - 1]++; }
	std::memcpy(buf + 9, hist, 8);
	uint32_t pos = 17;
	for (const auto& s : t.syms) {
		for (uint32_t j = 0; j < s.len; ++j) { buf[pos++] = static_cast<uint8_t>(s.val >> (8 * j)); }
	}
	return pos;
}

void compress_string(const SymTable& t, const uint8_t* s, uint32_t n, std::vector<uint8_t>* out) {
	uint32_t p = 0;
	while (p < n) {
		uint32_t  len  = 1;
		const int code = t.match(s + p, n - p, &len);
		if (code >= 0) {
			out->push_back(static_cast<uint8_t>(code));
			p += len;
		} else {
			out->push_back(255);
			out->push_back(s[p]);
			p += 1;
		}
	}
}

cudaStream_t enc_stream() {
	static cudaStream_t s[64] {};
	int                 d = 0;
	if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) { return nullptr; }
	if (!s[d]) { cudaStreamCreateWithFlags(&s[d], cudaStreamNonBlocking); }
	return s[d];
}

struct DBuf {
	void*        p = nullptr;
	cudaStream_t s;
	explicit DBuf(cudaStream_t st) : s(st) {}
	bool alloc(size_t n) { return cudaMallocAsync(&p, n ? n : 16, s) == cudaSuccess; }
	~DBuf() {
		if (p) { cudaFreeAsync(p, s); }
	}
};

// RLE DELTA_NO_PATCH page for T = uint32_t / uint64_t
template <class T>
int encode_rle(const T* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size, uint64_t* mtd_size) {
	const uint64_t n_vec = n / 1024;
	if (n_vec > 0xFFFFu) { return FLS_ERR_ARG; }
	cudaStream_t s = enc_stream();
	if (!s) { return FLS_ERR_CUDA; }
	std::vector<uint16_t> idx(n_vec * 1024);
	std::vector<T>        vals;
	std::vector<uint64_t> val_off(n_vec + 1, 0);
	vals.reserve(n_vec * 128);
	for (uint64_t v = 0; v < n_vec; ++v) {
		const T* x    = in + v * 1024;
		uint16_t pos  = 0;
		val_off[v]    = vals.size() * sizeof(T);
		vals.push_back(x[0]);
		idx[v * 1024] = 0;
		for (uint32_t i = 1; i < 1024; ++i) {
			if (x[i] != x[i - 1]) {
				vals.push_back(x[i]);
				++pos;
			}
			idx[v * 1024 + i] = pos;
		}
	}
	val_off[n_vec] = vals.size() * sizeof(T);
	std::vector<uint8_t>  bw(n_vec);
	std::vector<uint16_t> base(n_vec);
	std::vector<uint16_t> lane_bases(n_vec * 64);
	std::vector<uint64_t> off(n_vec);
	uint64_t              packed_total = 0;
	DBuf                  d_idx(s), d_tr(s), d_delta(s), d_bw(s), d_base(s), d_off(s), d_packed(s);
	if (n_vec) {
		const uint64_t b16 = n_vec * 1024 * 2;
		if (!d_idx.alloc(b16) || !d_tr.alloc(b16) || !d_delta.alloc(b16) || !d_bw.alloc(n_vec) ||
		    !d_base.alloc(n_vec * 2) || !d_off.alloc(n_vec * 8)) {
			return FLS_ERR_CUDA;
		}
		cudaMemcpyAsync(d_idx.p, idx.data(), b16, cudaMemcpyHostToDevice, s);
		int rc = fls_gpu_transpose_i_u16(static_cast<uint16_t*>(d_idx.p), static_cast<uint16_t*>(d_tr.p), n_vec, s);
		if (rc != FLS_OK) { return rc; }
		cudaMemcpy2DAsync(lane_bases.data(), 128, d_tr.p, 2048, 128, n_vec, cudaMemcpyDeviceToHost, s);
		rc = fls_gpu_unrsum_u16(static_cast<uint16_t*>(d_tr.p), static_cast<uint16_t*>(d_delta.p), n_vec, s);
		if (rc != FLS_OK) { return rc; }
		rc = fls_gpu_analyze_u16(static_cast<uint16_t*>(d_delta.p), static_cast<uint8_t*>(d_bw.p),
		                         static_cast<uint16_t*>(d_base.p), n_vec, 0, s);
		if (rc != FLS_OK) { return rc; }
		cudaMemcpyAsync(bw.data(), d_bw.p, n_vec, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(base.data(), d_base.p, n_vec * 2, cudaMemcpyDeviceToHost, s);
		if (cudaStreamSynchronize(s) != cudaSuccess) { return FLS_ERR_CUDA; }
		for (uint64_t v = 0; v < n_vec; ++v) {
			off[v] = packed_total;
			packed_total += bw[v] * 128ull;
		}
		if (!d_packed.alloc(packed_total + 16)) { return FLS_ERR_CUDA; }
		cudaMemcpyAsync(d_off.p, off.data(), n_vec * 8, cudaMemcpyHostToDevice, s);
		rc = fls_gpu_ffor_u16(static_cast<uint16_t*>(d_delta.p), static_cast<uint16_t*>(d_packed.p),
		                      static_cast<uint8_t*>(d_bw.p), static_cast<uint16_t*>(d_base.p),
		                      static_cast<uint64_t*>(d_off.p), n_vec, s);
		if (rc != FLS_OK) { return rc; }
	}
	const uint32_t arr_c = 5;
	const uint64_t len[5] = {vals.size() * sizeof(T), n_vec * 128, n_vec, n_vec * 2, packed_total};
	const uint64_t meta   = 8 + 4ull * arr_c + 4ull * arr_c * (n_vec ? n_vec - 1 : 0);
	uint64_t       total  = meta;
	for (auto l : len) { total += l; }
	if (out_size) { *out_size = total; }
	if (mtd_size) { *mtd_size = meta; }
	if (!out || total > cap) {
		cudaStreamSynchronize(s);
		return FLS_ERR_ARG;
	}
	std::memset(out, 0, 8);
	out[0]               = 6; // RLE
	out[1]               = 2; // DELTA_NO_PATCH
	const uint16_t vec_c = static_cast<uint16_t>(n_vec);
	std::memcpy(out + 4, &vec_c, 2);
	uint64_t boff[5];
	boff[0] = meta;
	for (int i = 1; i < 5; ++i) { boff[i] = boff[i - 1] + len[i - 1]; }
	for (uint32_t i = 0; i < arr_c; ++i) {
		const uint32_t o = static_cast<uint32_t>(boff[i]);
		std::memcpy(out + 8 + 4 * i, &o, 4);
	}
	for (uint64_t v = 1; v < n_vec; ++v) {
		const uint32_t e[5] = {static_cast<uint32_t>(val_off[v]), static_cast<uint32_t>(v * 128),
		                       static_cast<uint32_t>(v), static_cast<uint32_t>(v * 2), static_cast<uint32_t>(off[v])};
		std::memcpy(out + 8 + 4 * arr_c + 4ull * arr_c * (v - 1), e, 4 * arr_c);
	}
	if (!vals.empty()) { std::memcpy(out + boff[0], vals.data(), len[0]); }
	if (n_vec) {
		std::memcpy(out + boff[1], lane_bases.data(), len[1]);
		std::memcpy(out + boff[2], bw.data(), len[2]);
		std::memcpy(out + boff[3], base.data(), len[3]);
		cudaMemcpyAsync(out + boff[4], d_packed.p, packed_total, cudaMemcpyDeviceToHost, s);
	}
	return cudaStreamSynchronize(s) == cudaSuccess ? FLS_OK : FLS_ERR_CUDA;
}

} // namespace

int encode_rle_page(const void* in, uint64_t n, uint64_t cap, uint8_t* out, uint64_t* out_size, uint64_t* mtd_size,
                    int width) {
	return width == 64 ? encode_rle(static_cast<const uint64_t*>(in), n, cap, out, out_size, mtd_size)
	                   : encode_rle(static_cast<const uint32_t*>(in), n, cap, out, out_size, mtd_size);
}

} // namespace flsgpu

using namespace flsgpu;

extern "C" {

int fls_fsst_compress(const uint8_t* bytes, const uint64_t* offsets, uint64_t n, uint8_t* table_out,
                      uint64_t table_cap, uint64_t* table_size, uint8_t* comp_out, uint64_t comp_cap,
                      uint64_t* comp_offsets) {
	if ((!bytes && n) || !offsets || !table_out || !table_size || (!comp_out && comp_cap) || !comp_offsets) {
		return FLS_ERR_ARG;
	}
	std::vector<std::pair<const uint8_t*, uint32_t>> sample;
	sample.reserve(n);
	for (uint64_t i = 0; i < n; ++i) {
		if (offsets[i + 1] < offsets[i]) { return FLS_ERR_ARG; }
		sample.push_back({bytes + offsets[i], static_cast<uint32_t>(offsets[i + 1] - offsets[i])});
	}
	const SymTable t = build_table(sample);
	uint8_t        tb[8 + 1 + 8 + 2048 + 1];
	const uint32_t tl = export_table(t, tb);
	*table_size       = tl;
	if (tl > table_cap) { return FLS_ERR_ARG; }
	std::memcpy(table_out, tb, tl);
	std::vector<uint8_t> comp;
	comp_offsets[0] = 0;
	for (uint64_t i = 0; i < n; ++i) {
		compress_string(t, sample[i].first, sample[i].second, &comp);
		comp_offsets[i + 1] = comp.size();
	}
	if (comp.size() > comp_cap) { return FLS_ERR_ARG; }
	if (!comp.empty()) { std::memcpy(comp_out, comp.data(), comp.size()); }
	return FLS_OK;
}

int fls_encode_string_dict(const uint8_t* dict_bytes, const uint64_t* dict_offsets, uint32_t n_dict,
                           const uint32_t* codes, uint64_t n_rows, uint8_t* page_out, uint64_t page_cap,
                           uint64_t* page_size, uint8_t* dict_out, uint64_t dict_cap, uint64_t* dict_size) {
	if (!dict_offsets || n_dict == 0 || !codes || !page_size || !dict_size) { return FLS_ERR_ARG; }
	for (uint64_t i = 0; i < n_rows / 1024 * 1024; ++i) {
		if (codes[i] >= n_dict) { return FLS_ERR_ARG; }
	}
	// dictionary page
	std::vector<uint8_t>  table(8 + 1 + 8 + 2048 + 1);
	std::vector<uint64_t> coffs(n_dict + 1);
	const uint64_t        raw = dict_offsets[n_dict] - dict_offsets[0];
	std::vector<uint8_t>  comp(2 * raw + 16);
	uint64_t              tl = 0;
	int rc = fls_fsst_compress(dict_bytes, dict_offsets, n_dict, table.data(), table.size(), &tl, comp.data(),
	                           comp.size(), coffs.data());
	if (rc != FLS_OK) { return rc; }
	const uint64_t slot  = 8 + 1 + 8 + 2048 + 1; // FSST_MAXHEADER
	const uint64_t dsize = 8 + slot + 4ull * n_dict + coffs[n_dict];
	*dict_size           = dsize;
	if (!dict_out || dsize > dict_cap) { return FLS_ERR_ARG; }
	std::memset(dict_out, 0, 8 + slot);
	dict_out[0] = 8; // dict_hdr_t.exp_t = DICT
	std::memcpy(dict_out + 4, &n_dict, 4);
	std::memcpy(dict_out + 8, table.data(), tl);
	for (uint32_t i = 0; i < n_dict; ++i) {
		const uint32_t l = static_cast<uint32_t>(coffs[i + 1] - coffs[i]);
		std::memcpy(dict_out + 8 + slot + 4ull * i, &l, 4);
	}
	if (coffs[n_dict]) { std::memcpy(dict_out + 8 + slot + 4ull * n_dict, comp.data(), coffs[n_dict]); }
	// codes page: a u32 FFOR page under the DICT FFOR_NO_PATCH header
	uint64_t mtd = 0;
	rc = fls_encode_from_memory_status(const_cast<uint32_t*>(codes), n_rows, page_cap, page_out, page_size, &mtd,
	                                   UINT32, 1);
	if (rc != FLS_OK) { return rc; }
	page_out[0] = 8; // DICT
	page_out[1] = 2; // FFOR_NO_PATCH
	return FLS_OK;
}

int fls_encode_int_dict(const void* in, uint64_t n, int width, int rle, uint8_t* page_out, uint64_t page_cap,
                        uint64_t* page_size, uint8_t* dict_out, uint64_t dict_cap, uint64_t* dict_size) {
	if (!in || !page_size || !dict_size || (width != 32 && width != 64)) { return FLS_ERR_ARG; }
	n = n / 1024 * 1024;
	// dictionary in first-occurrence order (src/cor/lyt/dic/dic_fac.cpp:19-40)
	std::vector<uint32_t> codes(n);
	std::vector<uint64_t> entries;
	{
		std::unordered_map<uint64_t, uint32_t> idx;
		idx.reserve(n / 4 + 16);
		for (uint64_t i = 0; i < n; ++i) {
			const uint64_t x = width == 64 ? static_cast<const uint64_t*>(in)[i] : static_cast<const uint32_t*>(in)[i];
			auto           r = idx.emplace(x, static_cast<uint32_t>(entries.size()));
			if (r.second) { entries.push_back(x); }
			codes[i] = r.first->second;
		}
	}
	const uint64_t sz    = width / 8;
	const uint64_t raw   = entries.size() * sz;
	const uint64_t dsize = 8 + 12 + raw;
	*dict_size           = dsize;
	if (!dict_out || dsize > dict_cap) { return FLS_ERR_ARG; }
	// dict_hdr_t (include/fls/cor/lyt/dic/dic.hpp:32-41), then a rec buffer holding the entries raw: rec_hdr
	// {bw 255, pad, exc_c 0, base = byte count} (include/fls/cor/lyt/rec_hdr.hpp:7-13)
	std::memset(dict_out, 0, 20);
	dict_out[0]             = 8; // DICT
	const uint32_t entry_c  = static_cast<uint32_t>(entries.size());
	std::memcpy(dict_out + 4, &entry_c, 4);
	dict_out[8] = 255;
	std::memcpy(dict_out + 12, &raw, 8);
	for (uint64_t e = 0; e < entries.size(); ++e) {
		if (width == 64) {
			std::memcpy(dict_out + 20 + 8 * e, &entries[e], 8);
		} else {
			const uint32_t x = static_cast<uint32_t>(entries[e]);
			std::memcpy(dict_out + 20 + 4 * e, &x, 4);
		}
	}
	uint64_t mtd = 0;
	int      rc;
	if (rle) {
		// DICT_RLE DELTA_NO_PATCH: the RLE page layout over the u32 codes
		rc = encode_rle_page(codes.data(), n, page_cap, page_out, page_size, &mtd, 32);
		if (rc != FLS_OK) { return rc; }
		page_out[0] = 11; // DICT_RLE, variant 2 kept
	} else {
		rc = fls_encode_from_memory_status(codes.data(), n, page_cap, page_out, page_size, &mtd, UINT32, 1);
		if (rc != FLS_OK) { return rc; }
		page_out[0] = 8; // DICT
		page_out[1] = 2; // FFOR_NO_PATCH
	}
	return FLS_OK;
}

} // extern "C"
