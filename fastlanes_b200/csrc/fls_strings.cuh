// String decoding on the B200: FSST symbol tables, dictionary pages and string columns.
//
// Reference semantics (cwida/FastLanes):
//   * FSST decode (include/fls/cor/prm/fsst/fsst.h:152-259): code < 255 emits its symbol (len[code] bytes,
//     little-endian in a 64-bit word), 255 escapes the next byte.
//   * string dictionary page (src/cor/lyt/dic/dic.cpp:88-111, src/cor/eng/hzl_de_cmp.cpp:85-117):
//     dict_hdr_t (8 B) | FSST table (FSST_MAXHEADER = 2066 B slot) | entry_c x u32 compressed lengths |
//     compressed bytes; entry i decodes from the bytes after entries 0..i-1; UNFSST keeps cumulative END
//     offsets of the decoded entries.
//   * DICT / DICT_RLE rows (include/fls/encoder/assert_eq.hpp:257-400): row i is dictionary entry code[i],
//     codes untransposed (and RLE-expanded for DICT_RLE).
//   * FSST column (include/fls/encoder/assert_eq.hpp:166-210, src/cor/lyt/vec.cpp:162-207): per vector the
//     compressed bytes and 1024 cumulative end offsets (transposed); row i decodes bytes [end[i-1], end[i]).
//   * FSST12 (include/fls/cor/prm/fsst12/fsst12.h:130-177, src/cor/lyt/vec.cpp:208-248): the same column
//     layout; every 3 compressed bytes hold two 12-bit codes (bits 0-11, 12-23, little-endian), a trailing
//     2 bytes one code; no escapes.
// Output is Arrow-style: n_rows + 1 u32 offsets and the concatenated bytes.
#pragma once

#include "fls_device.cuh"
#include "fls_plan.h"
#include "fls_strplan.h"

namespace flsgpu {

// Decoded length of one FSST-compressed string.
__device__ __forceinline__ uint32_t fsst_decoded_len(const uint8_t* len, const uint8_t* in, uint32_t n) {
	uint32_t out = 0;
	for (uint32_t i = 0; i < n; ++i) {
		const uint8_t c = in[i];
		if (c == 255) {
			out += 1;
			++i;
		} else {
			out += len[c];
		}
	}
	return out;
}

// Decode one FSST-compressed string to out (exactly the decoded length is written).
__device__ __forceinline__ void fsst_decode_to(const uint64_t* sym, const uint8_t* len, const uint8_t* in, uint32_t n,
                                               uint8_t* out) {
	uint32_t o = 0;
	for (uint32_t i = 0; i < n; ++i) {
		const uint8_t c = in[i];
		if (c == 255) {
			if (i + 1 < n) { out[o] = in[i + 1]; }
			o += 1;
			++i;
		} else {
			const uint64_t s = sym[c];
			const uint32_t l = len[c];
			for (uint32_t b = 0; b < l; ++b) { out[o + b] = static_cast<uint8_t>(s >> (8 * b)); }
			o += l;
		}
	}
}

// Write the n bytes at byte offset `start` of the 4-byte aligned word array `base` to the window at byte offset
// d.  Every window word is stored whole by the row that owns its first byte (bytes past that row's end are
// zero in the store); a row that starts inside a word instead returns its bytes of that word (*head, word
// *hk), for an atomic OR once every lane's stores are done.  So the window needs no zeroing, only the word
// that the first row of a run of batches starts inside must hold zeros past the filled bytes.  Only the source
// words that hold bytes of the row are read.  Returns whether a head is left to OR.
__device__ __forceinline__ bool put_row(uint32_t* __restrict__ win, uint32_t d, const uint32_t* __restrict__ base,
                                        uint32_t start, uint32_t n, uint32_t* hk, uint32_t* head) {
	// the row is bytes [start, start + n) of the word array `base`; word indices (not pointers) keep the array's
	// address space (shared memory for a dictionary held there)
	if (n == 0) { return false; }
	const int32_t  a    = static_cast<int32_t>(start) - static_cast<int32_t>(d & 3u); // lands on window byte 4*(d/4)
	const uint32_t sh   = 8u * (static_cast<uint32_t>(a) & 3u);
	const int32_t  s    = a >> 2;
	const int32_t  s_lo = static_cast<int32_t>(start >> 2);
	const int32_t  s_hi = static_cast<int32_t>((start + n - 1) >> 2);
	const uint32_t k0 = d >> 2, k1 = (d + n - 1) >> 2;
	const uint32_t hm = 0xFFFFFFFFu << (8u * (d & 3u));
	const uint32_t tm = 0xFFFFFFFFu >> (8u * (3u - ((d + n - 1) & 3u)));
	// a clamped word only feeds bytes outside the row, which the masks drop
	uint32_t       w0  = base[s < s_lo ? s_lo : s];
	uint32_t       w1  = base[s + 1 > s_hi ? s_hi : s + 1];
	const uint32_t h   = __funnelshift_r(w0, w1, sh) & hm & (k0 == k1 ? tm : 0xFFFFFFFFu);
	const bool     mid = (d & 3u) != 0;
	if (!mid) { win[k0] = h; }
	*hk   = k0;
	*head = h;
	if (k0 == k1) { return mid; }
	const uint32_t m = k1 - k0; // words k0 + 1 .. k1 - 1 are whole row words
	uint32_t       j = 1;
#pragma unroll 4
	for (; j < m; ++j) {
		w0          = w1;
		w1          = base[s + static_cast<int32_t>(j) + 1];
		win[k0 + j] = __funnelshift_r(w0, w1, sh);
	}
	w0                = w1;
	const int32_t lst = s + static_cast<int32_t>(m) + 1;
	w1                = base[lst > s_hi ? s_hi : lst];
	win[k1]           = __funnelshift_r(w0, w1, sh) & tm;
	return mid;
}

// Decode one FSST-compressed string into the word array `win` at byte offset d, whole 32-bit words: the
// decoded bytes gather in a bit accumulator and leave as word stores, every word stored by the row that owns
// its first byte, bytes past the row's end zero (the protocol of the string kernels' window).  A row that
// starts inside a word returns its bytes of that word instead (*hk, *head) for an atomic OR once every lane's
// stores are done.  The bytes are those of fsst_decode_to, an escape at the string's end giving a zero byte.
__device__ __forceinline__ bool fsst_put_row(uint32_t* win, uint32_t d, const uint64_t* sym, const uint8_t* len,
                                             const uint8_t* in, uint32_t n, uint32_t* hk, uint32_t* head) {
	const uint32_t k0  = d >> 2;
	const bool     mid = (d & 3u) != 0;
	uint32_t       k   = k0;
	uint32_t       nb  = 8u * (d & 3u); // bits of word k below the next byte (earlier rows' bytes stay zero)
	uint64_t       acc = 0;             // bits of words k, k + 1 (byte 4k at bit 0)
	uint32_t       hi  = 0;             // bits of word k + 2
	bool           any = false, held = false;
	auto emit = [&](uint32_t w) {
		if (k == k0 && mid) {
			*hk  = k;
			*head = w;
			held  = true;
		} else {
			win[k] = w;
		}
		++k;
	};
	for (uint32_t i = 0; i < n; ++i) {
		const uint8_t c = in[i];
		uint64_t      s;
		uint32_t      l;
		if (c == 255) {
			s = i + 1 < n ? in[i + 1] : 0u;
			l = 1;
			++i;
		} else {
			s = sym[c];
			l = len[c];
		}
		if (l == 0) { continue; }
		any = true;
		// nb < 32 here: the symbol's up to 64 bits land in bits [nb, nb + 8l) of acc and hi
		acc |= s << nb;
		if (nb) { hi |= static_cast<uint32_t>(s >> (64u - nb)); }
		nb += 8u * l;
		while (nb >= 32u) {
			emit(static_cast<uint32_t>(acc));
			acc = (acc >> 32) | (static_cast<uint64_t>(hi) << 32);
			hi  = 0;
			nb -= 32u;
		}
	}
	if (any && nb > 8u * ((k == k0) ? (d & 3u) : 0u)) { emit(static_cast<uint32_t>(acc)); }
	return held;
}

// Decoded length of one FSST12-compressed string.  A trailing single byte (which the encoder never writes)
// decodes as the code of its 8 bits; the reference's decoder reads the byte after the string there.
__device__ __forceinline__ uint32_t fsst12_decoded_len(const uint8_t* len, const uint8_t* in, uint32_t n) {
	uint32_t out = 0, i = 0;
	for (; i + 3 <= n; i += 3) {
		const uint32_t c = in[i] | (static_cast<uint32_t>(in[i + 1]) << 8) | (static_cast<uint32_t>(in[i + 2]) << 16);
		out += len[c & 4095u] + len[c >> 12];
	}
	if (i < n) { out += len[(in[i] | (i + 1 < n ? static_cast<uint32_t>(in[i + 1]) << 8 : 0u)) & 4095u]; }
	return out;
}

__device__ __forceinline__ uint32_t fsst12_emit(const uint64_t* sym, const uint8_t* len, uint32_t code, uint8_t* out) {
	const uint64_t s = sym[code];
	const uint32_t l = len[code];
	for (uint32_t b = 0; b < l; ++b) { out[b] = static_cast<uint8_t>(s >> (8 * b)); }
	return l;
}

// Decode one FSST12-compressed string to out (exactly the decoded length is written).
__device__ __forceinline__ void fsst12_decode_to(const uint64_t* sym, const uint8_t* len, const uint8_t* in,
                                                 uint32_t n, uint8_t* out) {
	uint32_t o = 0, i = 0;
	for (; i + 3 <= n; i += 3) {
		const uint32_t c = in[i] | (static_cast<uint32_t>(in[i + 1]) << 8) | (static_cast<uint32_t>(in[i + 2]) << 16);
		o += fsst12_emit(sym, len, c & 4095u, out + o);
		o += fsst12_emit(sym, len, c >> 12, out + o);
	}
	if (i < n) { fsst12_emit(sym, len, (in[i] | (i + 1 < n ? static_cast<uint32_t>(in[i + 1]) << 8 : 0u)) & 4095u, out + o); }
}

// Inclusive warp scan (Kogge-Stone over shuffles).
template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T x, uint32_t lane) {
#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const T y = __shfl_up_sync(0xFFFFFFFFu, x, d);
		if (lane >= static_cast<uint32_t>(d)) { x += y; }
	}
	return x;
}

template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
	for (int d = 16; d > 0; d >>= 1) { x += __shfl_xor_sync(0xFFFFFFFFu, x, d); }
	return x;
}

} // namespace flsgpu
