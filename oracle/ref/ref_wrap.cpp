// Test infrastructure only: a flat extern "C" face over the reference's own C++ code, so that Python tests
// can drive it through ctypes.  It is linked into oracle/_ref/libfls_ref.so together with the reference
// sources; nothing in the product links it.
//
// Primitive wrappers call generated::<op>::fallback::scalar::<op> (include/fls_gen/*).
// Column wrappers follow the reference's own encode-and-verify driver
// (src/encoder/exp_col_encoder.cpp:40-64) and its materialisation rules, which live in the verifier
// include/fls/encoder/assert_eq.hpp:50-400 (untranspose for FFOR/DELTA, flatten+untranspose for RLE,
// untranspose+gather for DICT, flatten+untranspose+gather for DICT_RLE, per-row fsst_decompress for FSST).
// For string dictionaries the gather uses the end offsets that HzlDeCmp::UNFSST writes
// (src/cor/eng/hzl_de_cmp.cpp:85-117): entry i spans [end[i-1], end[i]).
#include "fastlanes.h"
#include "fls/cor/exp/exp_pool.hpp"
#include "fls/cor/lyt/buf.hpp"
#include "fls/cor/lyt/dic/dic.hpp"
#include "fls/cor/lyt/vec.hpp"
#include "fls/cor/prm/fsst/fsst.h"
#include "fls/cor/prm/fsst12/fsst12.h"
#include "fls/api/engine.hpp"
#include "fls/cor/eng/decompressor.hpp"
#include "fls/cor/eng/engine.hpp"
#include "fls/encoder/col_encoder.hpp"
#include "fls/encoder/exp_col_encoder.hpp"
#include "fls_gen/ffor/ffor.hpp"
#include "fls_gen/pack/pack.hpp"
#include "fls_gen/rsum/rsum.hpp"
#include "fls_gen/transpose/transpose.hpp"
#include "fls_gen/unffor/unffor.hpp"
#include "fls_gen/unpack/unpack.hpp"
#include "fls_gen/unrsum/unrsum.hpp"
#include "fls_gen/untranspose/untranspose.hpp"
#include "fls/connection.hpp"
#include "fls/expression/logical_expression.hpp"
#include "fls/expression/selection_ds.hpp"
#include "fls/primitive/predicate/equal.hpp"
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace fastlanes;
namespace gen = generated;

#define FLS_REF_PRIMS(T, S)                                                                                          \
	void ref_unpack_##S(const T* in, T* out, uint8_t bw) { gen::unpack::fallback::scalar::unpack(in, out, bw); }     \
	void ref_pack_##S(const T* in, T* out, uint8_t bw) { gen::pack::fallback::scalar::pack(in, out, bw); }           \
	void ref_unffor_##S(const T* in, T* out, uint8_t bw, const T* base) {                                          \
		gen::unffor::fallback::scalar::unffor(in, out, bw, base);                                                    \
	}                                                                                                                \
	void ref_ffor_##S(const T* in, T* out, uint8_t bw, const T* base) {                                            \
		gen::ffor::fallback::scalar::ffor(in, out, bw, base);                                                        \
	}                                                                                                                \
	void ref_rsum_##S(const T* in, T* out, const T* base) { gen::rsum::fallback::scalar::rsum(in, out, base); }     \
	void ref_unrsum_##S(const T* in, T* out) { gen::unrsum::fallback::scalar::unrsum(in, out); }                    \
	void ref_transpose_i_##S(const T* in, T* out) { gen::transpose::fallback::scalar::transpose_i(in, out); }      \
	void ref_untranspose_i_##S(const T* in, T* out) { gen::untranspose::fallback::scalar::untranspose_i(in, out); }

namespace {
Expression expression_of(const scheme_pool_t& pool, uint8_t expr_id, bool* ok) {
	auto it = pool.find(expr_id);
	if (it == pool.end()) {
		*ok = false;
		return Expression {};
	}
	*ok = true;
	return it->second;
}

int copy_out(const Buf& b, uint8_t* dst, uint64_t cap, uint64_t* sz) {
	*sz = b.Size();
	if (b.Size() > cap) { return -2; }
	if (b.Size() > 0) { std::memcpy(dst, b.data(), b.Size()); }
	return 0;
}

template <class PT>
int encode_col(const PT* data, uint64_t n, uint8_t expr_id, int verify, uint8_t* data_out, uint64_t data_cap,
               uint64_t* data_sz, uint8_t* dict_out, uint64_t dict_cap, uint64_t* dict_sz) {
	try {
		bool       ok  = false;
		Expression exp = expression_of(ExpPool<PT>::get_pool(), expr_id, &ok);
		if (!ok) { return -3; }
		std::vector<PT>   col(data, data + n);
		ExpColEncoder<PT> enc(verify != 0);
		ExpEncodedCol     res = enc.encode_pointer(col.data(), n, exp);
		int               rc  = copy_out(*res.data_buf, data_out, data_cap, data_sz);
		if (rc != 0) { return rc; }
		return copy_out(*res.dictionary_buf, dict_out, dict_cap, dict_sz);
	} catch (const std::exception&) { return -1; }
}

// Values come out as their 64-bit patterns, original order.
template <class PT>
int decode_col(const uint8_t* data, const uint8_t* dict, uint64_t dict_sz, uint64_t* out, uint64_t out_cap_vec,
               uint64_t* n_vec) {
	try {
		TColDecoder<PT> dec;
		if (dict_sz > 0) { dec.ExtInitDict(dict); }
		dec.InitDecompress(data);
		const n_t vc = dec.NVector();
		*n_vec       = vc;
		if (vc > out_cap_vec) { return -2; }
		const ExpT exp_t = static_cast<ExpT>(data[0]);
		for (n_t v = 0; v < vc; ++v) {
			Vec*      vec = dec.Decompress();
			uint64_t* o   = out + v * 1024;
			switch (exp_t) {
			case ExpT::UNCOMPRESSED:
			case ExpT::FFOR:
			case ExpT::DELTA:
				gen::untranspose::fallback::scalar::untranspose_i(
				    reinterpret_cast<const uint64_t*>(vec->buf_arr[0].data()), o);
				break;
			case ExpT::RLE: {
				uint64_t tr[1024];
				vec->flatten_to(tr);
				gen::untranspose::fallback::scalar::untranspose_i(tr, o);
				break;
			}
			case ExpT::DICT:
			case ExpT::DICT_FRQ:
			case ExpT::DICT_VAL: {
				auto*    idx_arr = reinterpret_cast<uint32_t*>(vec->buf_arr[vec->arr_c + 0].mutable_data());
				auto*    dic     = reinterpret_cast<const uint64_t*>(vec->dict_up->data_buf.mutable_data());
				uint32_t un[1024];
				gen::untranspose::fallback::scalar::untranspose_i(idx_arr, un);
				for (int i = 0; i < 1024; ++i) { o[i] = dic[un[i]]; }
				break;
			}
			case ExpT::DICT_RLE: {
				uint32_t tr[1024], un[1024];
				vec->flatten_to(tr);
				gen::untranspose::fallback::scalar::untranspose_i(tr, un);
				auto* dic = reinterpret_cast<const uint64_t*>(vec->dict_up->data_buf.mutable_data());
				for (int i = 0; i < 1024; ++i) { o[i] = dic[un[i]]; }
				break;
			}
			default:
				return -4;
			}
		}
		return 0;
	} catch (const std::exception&) { return -1; }
}
} // namespace

extern "C" {

FLS_REF_PRIMS(uint8_t, u8)
FLS_REF_PRIMS(uint16_t, u16)
FLS_REF_PRIMS(uint32_t, u32)
FLS_REF_PRIMS(uint64_t, u64)

/* Encode n int64 values (n a multiple of 1024) with pool expression expr_id (src/cor/exp_pool.cpp:22-61). */
int ref_encode_i64(const int64_t* data,
                   uint64_t       n,
                   uint8_t        expr_id,
                   int            verify,
                   uint8_t*       data_out,
                   uint64_t       data_cap,
                   uint64_t*      data_sz,
                   uint8_t*       dict_out,
                   uint64_t       dict_cap,
                   uint64_t*      dict_sz) {
	return encode_col<i64_pt>(data, n, expr_id, verify, data_out, data_cap, data_sz, dict_out, dict_cap, dict_sz);
}

/* The same for a double column (double pool, src/cor/exp_pool.cpp:104-137). */
int ref_encode_f64(const double* data,
                   uint64_t      n,
                   uint8_t       expr_id,
                   int           verify,
                   uint8_t*      data_out,
                   uint64_t      data_cap,
                   uint64_t*     data_sz,
                   uint8_t*      dict_out,
                   uint64_t      dict_cap,
                   uint64_t*     dict_sz) {
	return encode_col<dbl_pt>(data, n, expr_id, verify, data_out, data_cap, data_sz, dict_out, dict_cap, dict_sz);
}

/* Decode a reference-encoded int64 column to original order; *n_vec receives the vector count. */
int ref_decode_i64(const uint8_t* data,
                   const uint8_t* dict,
                   uint64_t       dict_sz,
                   int64_t*       out,
                   uint64_t       out_cap_vec,
                   uint64_t*      n_vec) {
	return decode_col<i64_pt>(data, dict, dict_sz, reinterpret_cast<uint64_t*>(out), out_cap_vec, n_vec);
}

/* The same for a double column (the values' bit patterns). */
int ref_decode_f64(const uint8_t* data,
                   const uint8_t* dict,
                   uint64_t       dict_sz,
                   double*        out,
                   uint64_t       out_cap_vec,
                   uint64_t*      n_vec) {
	return decode_col<dbl_pt>(data, dict, dict_sz, reinterpret_cast<uint64_t*>(out), out_cap_vec, n_vec);
}

/* Encode n strings given as Arrow-style (offsets[n+1], bytes) with string pool expression expr_id
 * (src/cor/exp_pool.cpp:66-101). */
int ref_encode_str(const uint8_t*  bytes,
                   const uint64_t* offsets,
                   uint64_t        n,
                   uint8_t         expr_id,
                   int             verify,
                   uint8_t*        data_out,
                   uint64_t        data_cap,
                   uint64_t*       data_sz,
                   uint8_t*        dict_out,
                   uint64_t        dict_cap,
                   uint64_t*       dict_sz) {
	try {
		bool       ok  = false;
		Expression exp = expression_of(ExpPool<str_pt>::get_pool(), expr_id, &ok);
		if (!ok) { return -3; }
		std::vector<std::string> col;
		col.reserve(n);
		for (uint64_t i = 0; i < n; ++i) {
			col.emplace_back(reinterpret_cast<const char*>(bytes + offsets[i]), offsets[i + 1] - offsets[i]);
		}
		ExpColEncoder<str_pt> enc(verify != 0);
		ExpEncodedCol         res = enc.encode_pointer(col.data(), n, exp);
		int                   rc  = copy_out(*res.data_buf, data_out, data_cap, data_sz);
		if (rc != 0) { return rc; }
		return copy_out(*res.dictionary_buf, dict_out, dict_cap, dict_sz);
	} catch (const std::exception&) { return -1; }
}

/* Decode a reference-encoded string column into Arrow-style offsets (u64, n_rows+1) + bytes. */
int ref_decode_str(const uint8_t* data,
                   const uint8_t* dict,
                   uint64_t       dict_sz,
                   uint8_t*       out_bytes,
                   uint64_t       bytes_cap,
                   uint64_t*      out_offsets,
                   uint64_t       rows_cap,
                   uint64_t*      n_rows) {
	try {
		TColDecoder<str_pt> dec;
		if (dict_sz > 0) { dec.ExtInitDict(dict); }
		dec.InitDecompress(data);
		const n_t  vc    = dec.NVector();
		const ExpT exp_t = static_cast<ExpT>(data[0]);
		*n_rows          = vc * 1024;
		if (vc * 1024 > rows_cap) { return -2; }
		uint64_t          pos = 0;
		std::vector<char> tmp(1 << 20);
		out_offsets[0] = 0;
		for (n_t v = 0; v < vc; ++v) {
			Vec* vec = dec.Decompress();
			switch (exp_t) {
			case ExpT::BYTE_ARR: {
				uint32_t un[1024];
				gen::untranspose::fallback::scalar::untranspose_i(vec->buf_arr[1].mutable_data<uint32_t>(), un);
				uint32_t start = 0;
				for (int i = 0; i < 1024; ++i) {
					const uint32_t len = un[i] - start;
					if (pos + len > bytes_cap) { return -2; }
					std::memcpy(out_bytes + pos, vec->buf_arr[0].data_at(start), len);
					pos += len;
					out_offsets[v * 1024 + i + 1] = pos;
					start                         = un[i];
				}
				break;
			}
			case ExpT::FSST: {
				auto*    str_p   = vec->buf_arr[vec->arr_c + 0].mutable_data();
				auto*    off_arr = vec->buf_arr[vec->arr_c + 1].mutable_data<uint32_t>();
				uint32_t un[1024];
				gen::untranspose::fallback::scalar::untranspose_i(off_arr, un);
				uint32_t start = 0;
				for (int i = 0; i < 1024; ++i) {
					const uint32_t len = un[i] - start;
					size_t         got = fsst_decompress(vec->fsst_decoder_up.get(), len, str_p + start, tmp.size(),
					                                     reinterpret_cast<unsigned char*>(tmp.data()));
					if (pos + got > bytes_cap) { return -2; }
					std::memcpy(out_bytes + pos, tmp.data(), got);
					pos += got;
					out_offsets[v * 1024 + i + 1] = pos;
					start                         = un[i];
				}
				break;
			}
			case ExpT::FSST12: {
				// as the FSST case, with the 12-bit decoder (include/fls/encoder/assert_eq.hpp:211-250)
				auto*    str_p   = vec->buf_arr[vec->arr_c + 0].mutable_data();
				auto*    off_arr = vec->buf_arr[vec->arr_c + 1].mutable_data<uint32_t>();
				uint32_t un[1024];
				gen::untranspose::fallback::scalar::untranspose_i(off_arr, un);
				uint32_t start = 0;
				for (int i = 0; i < 1024; ++i) {
					const uint32_t len = un[i] - start;
					size_t got = fsst12_decompress(vec->fsst12_decoder_up.get(), len, str_p + start, tmp.size(),
					                               reinterpret_cast<unsigned char*>(tmp.data()));
					if (pos + got > bytes_cap) { return -2; }
					std::memcpy(out_bytes + pos, tmp.data(), got);
					pos += got;
					out_offsets[v * 1024 + i + 1] = pos;
					start                         = un[i];
				}
				break;
			}
			case ExpT::DICT:
			case ExpT::DICT_FRQ:
			case ExpT::DICT_VAL:
			case ExpT::DICT_RLE: {
				uint32_t un[1024];
				if (exp_t == ExpT::DICT_RLE) {
					uint32_t tr[1024];
					vec->flatten_to(tr);
					gen::untranspose::fallback::scalar::untranspose_i(tr, un);
				} else {
					auto* idx_arr = reinterpret_cast<uint32_t*>(vec->buf_arr[vec->arr_c + 0].mutable_data());
					gen::untranspose::fallback::scalar::untranspose_i(idx_arr, un);
				}
				auto* byte_arr = vec->dict_up->data_buf.mutable_data();
				auto* ends     = reinterpret_cast<uint32_t*>(vec->dict_up->offs_buf.mutable_data());
				for (int i = 0; i < 1024; ++i) {
					const uint32_t idx   = un[i];
					const uint32_t start = idx == 0 ? 0 : ends[idx - 1];
					const uint32_t len   = ends[idx] - start;
					if (pos + len > bytes_cap) { return -2; }
					std::memcpy(out_bytes + pos, byte_arr + start, len);
					pos += len;
					out_offsets[v * 1024 + i + 1] = pos;
				}
				break;
			}
			default:
				return -4;
			}
		}
		return 0;
	} catch (const std::exception&) { return -1; }
}

/* The reference's C API (include/fastlanes.h:72-86), re-exported under distinct names so that the test process
 * can load this library and the product library side by side without symbol clashes. */
bool ref_encode_from_memory(void*     in,
                            uint64_t  n,
                            uint64_t  cap,
                            uint8_t*  out,
                            uint64_t* out_sz,
                            uint64_t* mtd_sz,
                            uint8_t   dt,
                            uint8_t   expr) {
	try {
		return encode_from_memory(in, n, cap, out, out_sz, mtd_sz, static_cast<data_t>(dt), expr);
	} catch (const std::exception&) { return false; }
}

int ref_decode_to_memory(uint8_t* enc, void* out, uint8_t dt) {
	try {
		decode_to_memory(enc, out, static_cast<data_t>(dt));
		return 0;
	} catch (const std::exception&) { return -1; }
}

/* FSST symbol-table import + decode of one string (include/fls/cor/prm/fsst/fsst.h:128-259). */
int64_t ref_fsst_decompress(const uint8_t* table, uint64_t in_len, const uint8_t* in, uint64_t cap, uint8_t* out) {
	fsst_decoder_t d;
	if (fsst_import(&d, const_cast<unsigned char*>(table)) == 0) { return -1; }
	return static_cast<int64_t>(fsst_decompress(&d, in_len, const_cast<unsigned char*>(in), cap, out));
}

/* Connection::read(dir).to_fls(out) (src/connection.cpp:25-56, :102-128): a CSV + schema.json directory to the
 * reference's file pair data.fls + footer.json.  Returns 0, or -1 when the reference throws. */
int ref_csv_to_fls(const char* in_dir, const char* out_dir) {
	try {
		fastlanes::Connection conn;
		conn.read(std::filesystem::path(in_dir)).to_fls(std::filesystem::path(out_dir));
		return 0;
	} catch (const std::exception&) { return -1; }
}

/* SelectionDS only keeps a reference to its LogicalExpr, which the predicate primitives never touch; the
 * reference defines no constructible LogicalExpr (src/expression/logical_expression.cpp has its member
 * definitions commented out), so the reference is bound to inert storage. */
static const LogicalExpr& no_expr() {
	alignas(LogicalExpr) static unsigned char raw[sizeof(LogicalExpr)] = {};
	return *reinterpret_cast<const LogicalExpr*>(raw);
}

/* The reference's predicate primitives on one decoded i64 vector (src/primitive/predicate/equal.cpp): op 0
 * eq_vector_constant_func (==), 1 ge_tvec_cvec (>), 2 lessthan_func (<).  The selected positions go to idx
 * (1024 u16); returns their count. */
int ref_predicate_i64(int op, const int64_t* vec, int64_t value, uint16_t* idx) {
	SelectionDS ds(no_expr());
	switch (op) {
	case 0: eq_vector_constant_func<i64_pt>(vec, value, ds); break;
	case 1: ge_tvec_cvec<i64_pt>(vec, &value, ds); break;
	case 2: lessthan_func<i64_pt>(vec, value, ds); break;
	default: return -1;
	}
	std::memcpy(idx, ds.idx_arr.data(), 1024 * sizeof(uint16_t));
	return ds.n_selected_values;
}

/* and_selection_ds_func (equal.cpp:100-119) of two index lists; returns the output count. */
int ref_selection_and(const uint16_t* i0, int n0, const uint16_t* i1, int n1, uint16_t* out) {
	SelectionDS a(no_expr()), b(no_expr()), c(no_expr());
	std::memcpy(a.idx_arr.data(), i0, sizeof(uint16_t) * n0);
	std::memcpy(b.idx_arr.data(), i1, sizeof(uint16_t) * n1);
	a.n_selected_values = static_cast<vec_idx_t>(n0);
	b.n_selected_values = static_cast<vec_idx_t>(n1);
	and_selection_ds_func(a, b, c);
	std::memcpy(out, c.idx_arr.data(), 1024 * sizeof(uint16_t));
	return c.n_selected_values;
}

} // extern "C"

#include <thread>

/* CPU baseline: the reference's own unffor (generated::unffor::fallback::scalar) over a batch of vectors,
 * split into contiguous vector ranges over n_threads std::threads (the reference itself is single-threaded;
 * the split is the benchmark's).  Vector v's packed words start at packed + byte_off[v]. */
extern "C" int ref_unffor_batch(int w, const uint8_t* packed, const uint64_t* byte_off, const uint8_t* bw,
                                const uint8_t* base, uint64_t n_vec, uint8_t* out, int n_threads) {
	if (n_threads < 1) { n_threads = 1; }
	auto work = [&](uint64_t lo, uint64_t hi) {
		for (uint64_t v = lo; v < hi; ++v) {
			const uint8_t* in = packed + byte_off[v];
			switch (w) {
			case 32:
				gen::unffor::fallback::scalar::unffor(reinterpret_cast<const uint32_t*>(in),
				                                      reinterpret_cast<uint32_t*>(out) + v * 1024, bw[v],
				                                      reinterpret_cast<const uint32_t*>(base) + v);
				break;
			case 64:
				gen::unffor::fallback::scalar::unffor(reinterpret_cast<const uint64_t*>(in),
				                                      reinterpret_cast<uint64_t*>(out) + v * 1024, bw[v],
				                                      reinterpret_cast<const uint64_t*>(base) + v);
				break;
			case 16:
				gen::unffor::fallback::scalar::unffor(reinterpret_cast<const uint16_t*>(in),
				                                      reinterpret_cast<uint16_t*>(out) + v * 1024, bw[v],
				                                      reinterpret_cast<const uint16_t*>(base) + v);
				break;
			default:
				gen::unffor::fallback::scalar::unffor(in, out + v * 1024, bw[v], base + v);
				break;
			}
		}
	};
	std::vector<std::thread> ts;
	const uint64_t           per = (n_vec + n_threads - 1) / n_threads;
	for (int t = 0; t < n_threads; ++t) {
		const uint64_t lo = t * per;
		const uint64_t hi = lo + per < n_vec ? lo + per : n_vec;
		if (lo >= hi) { break; }
		ts.emplace_back(work, lo, hi);
	}
	for (auto& t : ts) { t.join(); }
	return 0;
}

// The reference's column decode of FFOR vectors as decode_to_memory runs it (src/encoder/exp_col_decoder.cpp:13-26):
// per vector, the generated unffor into the vector buffer (ffor_decompress, src/cor/prm/ffor/ffor_decompress.cpp)
// then Materializer::Materialize's untranspose_i into the output (src/encoder/materializer.cpp:13-21): values in
// original order.  Vector ranges split over n_threads threads (the reference itself runs one).
template <typename T>
static void decode_ffor_range(const uint8_t* packed, const uint64_t* byte_off, const uint8_t* bw, const uint8_t* base,
                              uint64_t lo, uint64_t hi, uint8_t* out) {
	alignas(64) T vec[1024];
	for (uint64_t v = lo; v < hi; ++v) {
		gen::unffor::fallback::scalar::unffor(reinterpret_cast<const T*>(packed + byte_off[v]), vec, bw[v],
		                                      reinterpret_cast<const T*>(base) + v);
		gen::untranspose::fallback::scalar::untranspose_i(vec, reinterpret_cast<T*>(out) + v * 1024);
	}
}

extern "C" int ref_decode_ffor_batch(int w, const uint8_t* packed, const uint64_t* byte_off, const uint8_t* bw,
                                     const uint8_t* base, uint64_t n_vec, uint8_t* out, int n_threads) {
	if (w != 32 && w != 64) { return -1; }
	if (n_threads < 1) { n_threads = 1; }
	auto work = [&](uint64_t lo, uint64_t hi) {
		if (w == 32) {
			decode_ffor_range<uint32_t>(packed, byte_off, bw, base, lo, hi, out);
		} else {
			decode_ffor_range<uint64_t>(packed, byte_off, bw, base, lo, hi, out);
		}
	};
	std::vector<std::thread> ts;
	const uint64_t           per = (n_vec + n_threads - 1) / n_threads;
	for (int t = 0; t < n_threads; ++t) {
		const uint64_t lo = t * per;
		const uint64_t hi = lo + per < n_vec ? lo + per : n_vec;
		if (lo >= hi) { break; }
		ts.emplace_back(work, lo, hi);
	}
	for (auto& t : ts) { t.join(); }
	return 0;
}
