/* TEST INFRASTRUCTURE — CPU oracle for the FastLanes decode path (see fls_oracle.h).
 *
 * This file restates, in plain loops, what the reference's generated scalar primitives compute.  It is the
 * checker for the CUDA kernels and is never linked into the product.  Citations are to files of the
 * reference project (cwida/FastLanes); "scalar_aav_uf1/" abbreviates
 * primitives/fls_generated/fallback/scalar_aav_uf1/.
 */
#include "fls_oracle.h"

#include <string.h>

/* Unified transposed layout: transposed position k holds original index
 * (k % 16) * 64 + O[(k / 16) % 8] * 8 + k / 128 with O = {0,4,2,6,1,5,3,7}.  This is the permutation that
 * scalar_aav_uf1/fallback_scalar_aav_1024_uf1_transpose_src.cpp:4110 (u32) and :6162 (u64) spell out
 * element by element; transpose_o equals transpose_i. */
static const uint32_t FLS_O_ORDER[8] = {0, 4, 2, 6, 1, 5, 3, 7};

uint32_t fls_o_original_index(uint32_t k) {
	return (k % 16) * 64 + FLS_O_ORDER[(k / 16) % 8] * 8 + k / 128;
}

/* rsum chain of lane i: the W transposed positions i + L*j of that lane visited in ascending original index
 * (scalar_aav_uf1/fallback_scalar_aav_1024_uf1_rsum_src.cpp:100-205 for u32, :207-410 for u64). */
static void fls_o_chain(uint32_t width, uint32_t lane, uint32_t* chain) {
	const uint32_t L = 1024 / width;
	for (uint32_t j = 0; j < width; ++j) { chain[j] = lane + L * j; }
	/* insertion sort by original index; width <= 64 */
	for (uint32_t a = 1; a < width; ++a) {
		uint32_t x = chain[a];
		uint32_t b = a;
		while (b > 0 && fls_o_original_index(chain[b - 1]) > fls_o_original_index(x)) {
			chain[b] = chain[b - 1];
			--b;
		}
		chain[b] = x;
	}
}

#define FLS_O_DEFINE(T, S, W)                                                                                      \
	/* transpose_i: out[k] = in[orig(k)]  (scalar_aav_uf1/..._transpose_src.cpp) */                                  \
	void fls_o_transpose_i_##S(const T* in, T* out) {                                                              \
		for (uint32_t k = 0; k < 1024; ++k) { out[k] = in[fls_o_original_index(k)]; }                              \
	}                                                                                                              \
	/* untranspose_i: out[orig(k)] = in[k]  (scalar_aav_uf1/..._untranspose_src.cpp) */                              \
	void fls_o_untranspose_i_##S(const T* in, T* out) {                                                            \
		for (uint32_t k = 0; k < 1024; ++k) { out[fls_o_original_index(k)] = in[k]; }                              \
	}                                                                                                              \
	/* pack: value j of lane i goes to bits [j*bw, (j+1)*bw) of lane i's word stream in[i + L*w]                  \
	 * (scalar_aav_uf1/..._pack_src.cpp; inverse of unpack_src.cpp:1346-1420). bw == 0 writes nothing. */          \
	void fls_o_pack_##S(const T* in, T* out, uint8_t bw) {                                                         \
		const uint32_t L = 1024 / W;                                                                               \
		if (bw == 0) { return; }                                                                                   \
		for (uint32_t i = 0; i < L; ++i) {                                                                         \
			for (uint32_t w = 0; w < bw; ++w) { out[i + L * w] = 0; }                                              \
			for (uint32_t j = 0; j < W; ++j) {                                                                     \
				const uint64_t v   = (uint64_t)in[i + L * j];                                                      \
				const uint32_t bit = j * bw;                                                                       \
				for (uint32_t b = 0; b < bw; ++b) {                                                                \
					const uint32_t pos = bit + b;                                                                  \
					if ((v >> b) & 1u) { out[i + L * (pos / W)] |= (T)((T)1 << (pos % W)); }                       \
				}                                                                                                  \
			}                                                                                                      \
		}                                                                                                          \
	}                                                                                                              \
	/* unpack: inverse of pack; bw == 0 yields zeros (scalar_aav_uf1/..._unpack_src.cpp, u32 dispatch :17277). */   \
	void fls_o_unpack_##S(const T* in, T* out, uint8_t bw) {                                                       \
		const uint32_t L = 1024 / W;                                                                               \
		for (uint32_t i = 0; i < L; ++i) {                                                                         \
			for (uint32_t j = 0; j < W; ++j) {                                                                     \
				uint64_t       v   = 0;                                                                            \
				const uint32_t bit = j * bw;                                                                       \
				for (uint32_t b = 0; b < bw; ++b) {                                                                \
					const uint32_t pos = bit + b;                                                                  \
					v |= (uint64_t)((in[i + L * (pos / W)] >> (pos % W)) & 1u) << b;                               \
				}                                                                                                  \
				out[i + L * j] = (T)v;                                                                             \
			}                                                                                                      \
		}                                                                                                          \
	}                                                                                                              \
	/* ffor: pack(in - base) with wrap-around in T (scalar_aav_uf1/..._ffor_src.cpp). */                            \
	void fls_o_ffor_##S(const T* in, T* out, uint8_t bw, const T* base) {                                          \
		T tmp[1024];                                                                                               \
		for (uint32_t k = 0; k < 1024; ++k) { tmp[k] = (T)(in[k] - *base); }                                       \
		fls_o_pack_##S(tmp, out, bw);                                                                              \
	}                                                                                                              \
	/* unffor: unpack + base, wrap-around in T (scalar_aav_uf1/..._unffor_src.cpp, u32 :22971, body :1788). */      \
	void fls_o_unffor_##S(const T* in, T* out, uint8_t bw, const T* base) {                                        \
		fls_o_unpack_##S(in, out, bw);                                                                             \
		for (uint32_t k = 0; k < 1024; ++k) { out[k] = (T)(out[k] + *base); }                                      \
	}                                                                                                              \
	/* rsum: per-lane running sum along the lane's chain, seeded by base[lane]                                     \
	 * (scalar_aav_uf1/..._rsum_src.cpp:100-205 u32, :207-410 u64). */                                             \
	void fls_o_rsum_##S(const T* in, T* out, const T* base) {                                                      \
		const uint32_t L = 1024 / W;                                                                               \
		uint32_t       chain[64];                                                                                  \
		for (uint32_t i = 0; i < L; ++i) {                                                                         \
			fls_o_chain(W, i, chain);                                                                              \
			T acc = base[i];                                                                                       \
			for (uint32_t j = 0; j < W; ++j) {                                                                     \
				acc             = (T)(acc + in[chain[j]]);                                                         \
				out[chain[j]] = acc;                                                                               \
			}                                                                                                      \
		}                                                                                                          \
	}                                                                                                              \
	/* unrsum: first chain element becomes 0, every other one the difference to its chain predecessor           \
	 * (scalar_aav_uf1/..._unrsum_src.cpp:120-255 u32). */                                                         \
	void fls_o_unrsum_##S(const T* in, T* out) {                                                                   \
		const uint32_t L = 1024 / W;                                                                               \
		uint32_t       chain[64];                                                                                  \
		T              tmp[1024];                                                                                  \
		for (uint32_t i = 0; i < L; ++i) {                                                                         \
			fls_o_chain(W, i, chain);                                                                              \
			tmp[chain[0]] = 0;                                                                                     \
			for (uint32_t j = 1; j < W; ++j) { tmp[chain[j]] = (T)(in[chain[j]] - in[chain[j - 1]]); }             \
		}                                                                                                          \
		memcpy(out, tmp, sizeof(tmp));                                                                             \
	}                                                                                                              \
	/* analyze: base = min, bw = bits of (max - min) (src/cor/prm/ffor/ffor_analyze.cpp:77-102, which computes     \
	 * ceil(log2(delta + 1)) in double precision; this restatement counts bits exactly). */                       \
	uint8_t fls_o_analyze_##S(const T* in, T* base_out) {                                                          \
		T mn = in[0], mx = in[0];                                                                                  \
		for (uint32_t k = 1; k < 1024; ++k) {                                                                      \
			if (in[k] < mn) { mn = in[k]; }                                                                        \
			if (in[k] > mx) { mx = in[k]; }                                                                        \
		}                                                                                                          \
		uint64_t d  = (uint64_t)mx - (uint64_t)mn;                                                                 \
		uint8_t  bw = 0;                                                                                           \
		while (d) {                                                                                                \
			++bw;                                                                                                  \
			d >>= 1;                                                                                               \
		}                                                                                                          \
		*base_out = mn;                                                                                            \
		return bw;                                                                                                 \
	}                                                                                                              \
	/* Batch of vectors: vector v's packed words start at packed + word_off[v].  Output in transposed order        \
	 * (the primitive's own) or, with original_order, untransposed as Materializer::Materialize does              \
	 * (src/encoder/materializer.cpp:13-21). */                                                                    \
	void fls_o_unffor_batch_##S(const T* packed, const uint64_t* word_off, const uint8_t* bw, const T* base,      \
	                            uint64_t n_vec, int original_order, T* out) {                                      \
		T tmp[1024];                                                                                               \
		for (uint64_t v = 0; v < n_vec; ++v) {                                                                     \
			if (original_order) {                                                                                  \
				fls_o_unffor_##S(packed + word_off[v], tmp, bw[v], base + v);                                      \
				fls_o_untranspose_i_##S(tmp, out + v * 1024);                                                      \
			} else {                                                                                               \
				fls_o_unffor_##S(packed + word_off[v], out + v * 1024, bw[v], base + v);                           \
			}                                                                                                      \
		}                                                                                                          \
	}

FLS_O_DEFINE(uint8_t, u8, 8)
FLS_O_DEFINE(uint16_t, u16, 16)
FLS_O_DEFINE(uint32_t, u32, 32)
FLS_O_DEFINE(uint64_t, u64, 64)

/* fsst_import (src/cor/prm/fsst/libfsst.cpp:617-657): 8-byte version word whose upper 32 bits are 20190218,
 * byte 8 = zero-terminated flag, bytes 9..16 = lenHisto, then the symbol bytes grouped by length in the order
 * 2,3,4,5,6,7,8,1.  Codes are numbered from the flag value upward; unused codes decode to the 8-byte text
 * "corrupt\0". */
uint32_t fls_o_fsst_import(const uint8_t* buf, uint64_t* sym, uint8_t* len) {
	uint64_t version = 0;
	memcpy(&version, buf, 8);
	if ((version >> 32) != 20190218ull) { return 0; }
	const uint32_t zt = buf[8] & 1u;
	uint8_t        hist[8];
	memcpy(hist, buf + 9, 8);
	len[0]        = 1;
	sym[0]        = 0;
	uint32_t code = zt, pos = 17;
	if (zt) { hist[0]--; }
	for (uint32_t l = 1; l <= 8; ++l) {
		for (uint32_t i = 0; i < hist[l & 7]; ++i, ++code) {
			len[code] = (uint8_t)((l & 7) + 1);
			sym[code] = 0;
			for (uint32_t j = 0; j < len[code]; ++j) { sym[code] |= (uint64_t)buf[pos++] << (8 * j); }
		}
	}
	while (code < 255) {
		sym[code] = 32774747032022883ull;
		len[code] = 8;
		++code;
	}
	return pos;
}

/* fsst_decompress semantics (include/fls/cor/prm/fsst/fsst.h:152-259): code < 255 emits its symbol,
 * code 255 (escape) emits the next input byte verbatim.  The reference's 4-code fast path is an
 * optimisation of the same rule for well-formed input. */
uint64_t fls_o_fsst_decode(const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint64_t in_len, uint8_t* out,
                           uint64_t cap) {
	uint64_t pin = 0, pout = 0;
	while (pin < in_len) {
		const uint8_t code = in[pin++];
		if (code != 255) {
			for (uint32_t j = 0; j < len[code]; ++j, ++pout) {
				if (pout < cap) { out[pout] = (uint8_t)(sym[code] >> (8 * j)); }
			}
		} else {
			if (pin < in_len) {
				if (pout < cap) { out[pout] = in[pin]; }
				++pin;
			}
			++pout;
		}
	}
	return pout;
}

/* fsst12_import (src/cor/prm/fsst12/libfsst12.cpp:363-389): version word, 8 u16 symbol counts at byte 8, then
 * every symbol as a length byte and its bytes; unused codes are the 8 bytes "corrupt". */
uint32_t fls_o_fsst12_import(const uint8_t* buf, uint64_t avail, uint64_t* sym, uint8_t* len) {
	uint64_t version = 0, count = 0;
	if (avail < 24) { return 0; }
	memcpy(&version, buf, 8);
	if ((version >> 32) != 20190218ull) { return 0; }
	uint16_t hist[8];
	memcpy(hist, buf + 8, 16);
	for (int i = 0; i < 8; ++i) { count += hist[i]; }
	if (count > 4096) { return 0; }
	uint64_t pos = 24;
	for (uint64_t c = 0; c < count; ++c) {
		if (pos >= avail || buf[pos] > 8 || pos + 1 + buf[pos] > avail) { return 0; }
		len[c] = buf[pos++];
		sym[c] = 0;
		for (uint32_t j = 0; j < len[c]; ++j) { sym[c] |= (uint64_t)buf[pos++] << (8 * j); }
	}
	for (uint64_t c = count; c < 4096; ++c) {
		sym[c] = 32774747032022883ull;
		len[c] = 8;
	}
	return (uint32_t)pos;
}

static uint64_t fsst12_emit(const uint64_t* sym, const uint8_t* len, uint32_t code, uint8_t* out, uint64_t pout,
                            uint64_t cap) {
	for (uint32_t j = 0; j < len[code]; ++j) {
		if (pout + j < cap) { out[pout + j] = (uint8_t)(sym[code] >> (8 * j)); }
	}
	return pout + len[code];
}

uint64_t fls_o_fsst12_decode(const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint64_t in_len, uint8_t* out,
                             uint64_t cap) {
	uint64_t pin = 0, pout = 0;
	for (; pin + 3 <= in_len; pin += 3) {
		const uint32_t code = in[pin] | ((uint32_t)in[pin + 1] << 8) | ((uint32_t)in[pin + 2] << 16);
		pout = fsst12_emit(sym, len, code & 4095u, out, pout, cap);
		pout = fsst12_emit(sym, len, (code >> 12) & 4095u, out, pout, cap);
	}
	if (pin < in_len) {
		/* the encoder writes a lone code as 2 bytes; a lone trailing byte decodes as its own 8 bits */
		const uint32_t code = in[pin] | (pin + 1 < in_len ? (uint32_t)in[pin + 1] << 8 : 0u);
		pout = fsst12_emit(sym, len, code & 4095u, out, pout, cap);
	}
	return pout;
}

/* CPU baseline in the oracle port: the same batch decode as fls_o_unffor_batch_*, transposed order, for a
 * caller that splits vector ranges over threads itself. */
void fls_o_unffor_batch_bytes(int w, const uint8_t* packed, const uint64_t* byte_off, const uint8_t* bw,
                              const uint8_t* base, uint64_t lo, uint64_t hi, uint8_t* out) {
	for (uint64_t v = lo; v < hi; ++v) {
		const uint8_t* in = packed + byte_off[v];
		switch (w) {
		case 64: fls_o_unffor_u64((const uint64_t*)in, (uint64_t*)out + v * 1024, bw[v], (const uint64_t*)base + v); break;
		case 32: fls_o_unffor_u32((const uint32_t*)in, (uint32_t*)out + v * 1024, bw[v], (const uint32_t*)base + v); break;
		case 16: fls_o_unffor_u16((const uint16_t*)in, (uint16_t*)out + v * 1024, bw[v], (const uint16_t*)base + v); break;
		default: fls_o_unffor_u8(in, out + v * 1024, bw[v], base + v); break;
		}
	}
}
