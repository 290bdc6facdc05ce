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
	// four source words loaded before their four stores (more loads in flight); s + j + 4 <= s + m <= the
	// row's last source word
	for (; j + 3 < m; j += 4) {
		const int32_t  q  = s + static_cast<int32_t>(j);
		const uint32_t a1 = base[q + 1], a2 = base[q + 2], a3 = base[q + 3], a4 = base[q + 4];
		win[k0 + j]       = __funnelshift_r(w1, a1, sh);
		win[k0 + j + 1]   = __funnelshift_r(a1, a2, sh);
		win[k0 + j + 2]   = __funnelshift_r(a2, a3, sh);
		win[k0 + j + 3]   = __funnelshift_r(a3, a4, sh);
		w1                = a4;
	}
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

// ---------------------------------------------------------------------------------------------------------
// Code-parallel decode of one vector of an FSST (or BYTE_ARR) column, one warp.
//
// The rows of a vector are consecutive in its compressed bytes (row r is [end[r-1], end[r])), and FSST is
// context-free except for escapes, so the vector's bytes [0, end[1023]) decode as ONE stream whose output is the
// rows' bytes concatenated; row r's output offset is the decoded length of the stream before byte end[r-1].
// The warp walks the stream 128 bytes at a time, 4 bytes per lane:
//   * which bytes start a code: a byte is an escaped literal when the code before it is an escape (255); rows
//     restart the decoder (a row's first byte always starts a code).  Each lane composes the 2-state transfer
//     function of its 4 bytes (state 1 = "the next byte is a literal"), a warp scan of the functions gives every
//     lane its entry state.  Chunks without a 255 (nearly all of them) skip this: every byte starts a code.
//   * decoded lengths (symbol length; 1 for an escape; 0 for its literal) are prefix-summed across the warp;
//   * every lane writes its symbols at its offset into the warp's output window as whole words
//     (put_syms: the put_row protocol), and rows starting in the chunk take their offsets from the sums.
// An escape as a row's last byte decodes as one zero byte (as the oracle's row decoder does).
// ---------------------------------------------------------------------------------------------------------
constexpr uint32_t kStreamChunk = 128; // stream bytes per warp step

__device__ __forceinline__ uint32_t stream_row_start(const uint32_t* rows32, uint32_t r) {
	return r == 0 ? 0u : rows32[(r - 1) + ((r - 1) >> 5)];
}

// Escape-state transfer of one lane's bytes (bit j of esc: byte j is 255; of rs: a row starts at byte j; nv
// valid bytes): the state after them for entry state st.
__device__ __forceinline__ uint32_t esc_transfer(uint32_t st, uint32_t esc, uint32_t rs, uint32_t nv) {
#pragma unroll
	for (uint32_t j = 0; j < 4; ++j) {
		if (j < nv) {
			if ((rs >> j) & 1u) { st = 0; }
			st = st ? 0u : ((esc >> j) & 1u);
		}
	}
	return st;
}

// transfer functions as 2 bits, f(0) | f(1) << 1
__device__ __forceinline__ uint32_t fn_apply(uint32_t f, uint32_t x) { return (f >> x) & 1u; }
__device__ __forceinline__ uint32_t fn_compose(uint32_t later, uint32_t earlier) {
	return fn_apply(later, fn_apply(earlier, 0)) | (fn_apply(later, fn_apply(earlier, 1)) << 1);
}

// Row starts inside [cb, cb + 128): the 128-bit mask m (bit i: a row starts at byte cb + i) and whether a row
// starts at cb + 128.  *rc: on entry a row index at or before the first row starting at or after cb (rows
// before cb are skipped); on return the first row starting at or after cb + 128.
__device__ __forceinline__ void stream_row_mask(const uint32_t* rows32, uint32_t cb, uint32_t lane, uint32_t* rc,
                                                uint32_t m[4], bool* at_end) {
	m[0] = m[1] = m[2] = m[3] = 0;
	*at_end  = false;
	uint32_t r = *rc;
	while (r < kVec) {
		const uint32_t rr  = r + lane;
		const uint32_t s   = rr < kVec ? stream_row_start(rows32, rr) : 0xFFFFFFFFu;
		const bool     in  = s >= cb && s < cb + kStreamChunk;
		const uint32_t rel = s - cb;
#pragma unroll
		for (uint32_t k = 0; k < 4; ++k) {
			m[k] |= __reduce_or_sync(0xFFFFFFFFu, (in && (rel >> 5) == k) ? 1u << (rel & 31u) : 0u);
		}
		const uint32_t n = __popc(__ballot_sync(0xFFFFFFFFu, s < cb + kStreamChunk));
		r += n;
		if (n < 32) {
			*at_end = __any_sync(0xFFFFFFFFu, s == cb + kStreamChunk);
			break;
		}
	}
	*rc = r;
}

// A lane's decoded bytes -- up to 4 symbols (value, length; length 0 = nothing, its value then 0) in order --
// into the word window at byte d, whole words: every word is stored by the lane owning its first byte, bytes
// past the lane's end zero; a lane starting inside a word returns its bytes of that word (*hk, *head) for an
// atomic OR after a warp sync (the protocol of put_row).  Returns whether such a head is left.
// The bytes gather in a 128-bit accumulator a0..a3 (word k at a0) holding nb < 64 bits before every symbol, so
// a symbol (at most 64 bits) leaves at most one pair of whole words behind it: one predicated two-word emit
// per symbol, and no branch on where a word goes.
__device__ __forceinline__ bool put_syms(uint32_t* win, uint32_t d, const uint64_t (&sv)[4], const uint32_t (&sl)[4],
                                         uint32_t* hk, uint32_t* head) {
	const uint32_t k0  = d >> 2;
	const bool     mid = (d & 3u) != 0;
	uint32_t       k   = k0;
	uint32_t       nb  = 8u * (d & 3u);
	uint32_t       a0 = 0, a1 = 0, a2 = 0, a3 = 0;
	uint32_t       hv   = 0;
	bool           held = false;
	// words k, k + 1 leave: the first word of a lane that starts inside it is its head instead
	auto emit2 = [&]() {
		const bool h = mid && k == k0;
		if (!h) { win[k] = a0; }
		win[k + 1] = a1;
		hv         = h ? a0 : hv;
		held       = held || h;
	};
#pragma unroll
	for (int j = 0; j < 4; ++j) {
		const uint32_t lo = static_cast<uint32_t>(sv[j]), hi = static_cast<uint32_t>(sv[j] >> 32);
		const uint32_t sh = nb & 31u;
		const uint32_t t0 = lo << sh;
		const uint32_t t1 = __funnelshift_l(lo, hi, sh);
		const uint32_t t2 = __funnelshift_l(hi, 0u, sh); // hi >> (32 - sh), 0 for sh = 0
		const bool     lw = nb < 32u;
		a0 |= lw ? t0 : 0u;
		a1 |= lw ? t1 : t0;
		a2 |= lw ? t2 : t1;
		a3 |= lw ? 0u : t2;
		nb += 8u * sl[j];
		if (nb >= 64u) {
			emit2();
			a0 = a2;
			a1 = a3;
			a2 = 0;
			a3 = 0;
			k += 2;
			nb -= 64u;
		}
	}
	// what is left: bits [0, nb) of a0, a1 (nb > 8 * (d & 3) when the lane wrote nothing yet and has bytes)
	const bool any = (sl[0] | sl[1] | sl[2] | sl[3]) != 0;
	if (any && nb > 0u) {
		const bool h = mid && k == k0;
		if (!h) { win[k] = a0; }
		hv   = h ? a0 : hv;
		held = held || h;
		if (nb > 32u) { win[k + 1] = a1; }
	}
	*hk   = k0;
	*head = hv;
	return held;
}

// Compressed length of a vector's rows (rows32: its 1024 cumulative row end offsets, row r at word r + r / 32;
// vn: its compressed bytes): the last row's end.  *bad, and length 0, when the rows are not non-decreasing or
// end past vn.
__device__ __forceinline__ uint32_t stream_rows_length(const uint32_t* rows32, uint32_t vn, uint32_t lane, bool* bad) {
	uint32_t prev = lane == 0 ? 0u : rows32[(32 * lane - 1) + lane - 1];
	bool     b    = false;
#pragma unroll 8
	for (uint32_t i = 0; i < 32; ++i) {
		const uint32_t e = rows32[32 * lane + i + lane];
		b |= e < prev;
		prev = e;
	}
	b |= lane == 31 && prev > vn;
	*bad = __any_sync(0xFFFFFFFFu, b);
	return *bad ? 0u : rows32[kVec - 1 + (kVec - 1) / 32];
}

// Decoded byte total of an FSST vector's compressed bytes [0, L) when none of them is an escape (255): every
// byte is then a code and the total is the sum of their symbol lengths (len: the symbol lengths, code 255's 0).
// Returns false when a byte 255 may be among them -- the escape-aware walk (stream_vector) decides then; the
// zero-byte test can also fire on a byte 254 just above a 255 outside the range, which costs only that walk.
__device__ __forceinline__ bool fsst_plain_total(const uint8_t* vb, uint32_t L, const uint8_t* len, uint32_t lane,
                                                 uint32_t* total) {
	const uintptr_t va   = reinterpret_cast<uintptr_t>(vb);
	const uint32_t  off  = static_cast<uint32_t>(va & 3u);
	const uint32_t* base = reinterpret_cast<const uint32_t*>(va - off);
	const uint32_t  nw   = (off + L + 3u) >> 2; // words holding a byte of [0, L)
	uint32_t        sum = 0, esc = 0;
	// 8 words per lane in flight per round: the walk is one read of the bytes, bound by load latency otherwise
	constexpr uint32_t kU = 8;
	for (uint32_t q0 = lane; q0 < nw; q0 += 32 * kU) {
		uint32_t w[kU];
#pragma unroll
		for (uint32_t u = 0; u < kU; ++u) { w[u] = q0 + 32 * u < nw ? __ldg(base + q0 + 32 * u) : 0u; }
#pragma unroll
		for (uint32_t u = 0; u < kU; ++u) {
			const uint32_t q = q0 + 32 * u;
			if (q >= nw) { break; }
			const int64_t p0 = 4ll * q - off; // stream position of the word's byte 0
			uint32_t      vm;                 // 0x80 in every byte inside [0, L)
			if (p0 >= 0 && p0 + 4 <= static_cast<int64_t>(L)) {
				sum += len[w[u] & 0xFFu] + len[(w[u] >> 8) & 0xFFu] + len[(w[u] >> 16) & 0xFFu] + len[w[u] >> 24];
				vm = 0x80808080u;
			} else {
				vm = 0;
#pragma unroll
				for (uint32_t j = 0; j < 4; ++j) {
					const bool in = p0 + j >= 0 && p0 + j < static_cast<int64_t>(L);
					sum += in ? len[(w[u] >> (8 * j)) & 0xFFu] : 0u;
					vm |= in ? 0x80u << (8 * j) : 0u;
				}
			}
			const uint32_t x = ~w[u]; // escape bytes turn into zero bytes
			esc |= (x - 0x01010101u) & ~x & vm;
		}
	}
	*total = warp_sum(sum);
	return !__any_sync(0xFFFFFFFFu, esc != 0);
}

// Per-vector output of the materialising pass.
struct StreamOut {
	uint32_t* offsets;   // the vector's 1024 row offsets
	uint8_t*  bytes;     // output bytes (global)
	uint64_t  vbase;     // the vector's first output byte
	uint8_t*  win;       // the warp's kWindow-byte output window (shared memory, 16-byte aligned)
};

// One vector of an FSST (KIND_FSST = true) or BYTE_ARR column: rows32 its 1024 cumulative row end offsets in
// original order (row r at word r + r / 32), vb / vn its compressed bytes (vn 0 and rows all zero for none).
// Returns the decoded byte total; MAT also writes the offsets and bytes (o).  *bad: the rows are not
// non-decreasing within vn (the vector then decodes as 1024 empty rows).
template <bool MAT, bool KIND_FSST, uint32_t kWindow>
__device__ __forceinline__ uint32_t stream_vector(const uint32_t* rows32, const uint8_t* vb, uint32_t vn,
                                                  const uint64_t* sym, const uint8_t* len, uint32_t lane,
                                                  const StreamOut& o, bool* bad) {
	const uint32_t  L     = stream_rows_length(rows32, vn, lane, bad);
	if constexpr (!KIND_FSST && !MAT) { return L; } // a plain-bytes vector decodes to its own bytes
	const uintptr_t va    = reinterpret_cast<uintptr_t>(vb);
	const uint32_t  off   = static_cast<uint32_t>(va & 3u);
	const uint32_t* base  = reinterpret_cast<const uint32_t*>(va - off);
	const uint32_t  nw    = (off + L + 3u) >> 2; // words holding a byte of the stream [0, L)
	uint32_t*       win32 = reinterpret_cast<uint32_t*>(o.win);
	uint32_t        carry = 0; // 1: the chunk's first byte is an escaped literal
	uint32_t        vdec  = 0; // decoded bytes before the chunk
	uint32_t        rc    = 0; // first row whose offset is not written (MAT) / a row at or before cb (lengths)

	// window of the materialising pass: W = output position of win[0], fill bytes in it, lo = first output byte
	// it may write (the previous vector owns the bytes before vbase)
	uint64_t W    = o.vbase & ~15ull;
	uint32_t fill = static_cast<uint32_t>(o.vbase & 15u);
	uint64_t lo   = o.vbase;
	if constexpr (MAT) {
		// the first lane may start inside this word: it ORs its bytes in
		if (lane == 0) { win32[fill >> 2] = 0; }
		__syncwarp();
	}
	auto flush = [&](bool all) {
		const uint32_t full = fill & ~15u;
		const uint32_t upto = all ? fill : full;
		for (uint32_t c = 16 * lane; c < upto; c += 512) {
			const uint64_t g = W + c;
			if (g >= lo && c + 16 <= upto) {
				*reinterpret_cast<uint4*>(o.bytes + g) = *reinterpret_cast<const uint4*>(o.win + c);
			} else {
				for (uint32_t i = 0; i < 16 && c + i < upto; ++i) {
					if (g + i >= lo) { o.bytes[g + i] = o.win[c + i]; }
				}
			}
		}
		__syncwarp();
		if (!all) {
			// the partial chunk [full, fill) moves to the window start (its bytes past `fill` are zero: every word
			// was stored whole, zeros past its writer's end)
			if (lane == 0 && full != 0 && (fill & 15u) != 0) {
				*reinterpret_cast<uint4*>(o.win) = *reinterpret_cast<const uint4*>(o.win + full);
			}
			__syncwarp();
			W += full;
			fill &= 15u;
			lo = lo > W ? lo : W;
		}
	};

	// this lane's word of chunk j; loads run four chunks ahead of the decode (q0 = the current chunk's word)
	auto ldw = [&](uint32_t j) {
		const uint32_t q = j * (kStreamChunk / 4) + lane;
		return q < nw ? __ldg(base + q) : 0u;
	};
	uint32_t q0 = ldw(0), q1 = ldw(1), q2 = ldw(2), q3 = ldw(3);
	for (uint32_t cb = 0, ck = 0; cb < L; cb += kStreamChunk, ++ck) {
		const uint32_t w0   = q0;
		const uint32_t nxt  = __shfl_sync(0xFFFFFFFFu, q1, 0); // the word after the chunk: lane 0's of the next
		uint32_t       w1   = __shfl_down_sync(0xFFFFFFFFu, w0, 1);
		if (lane == 31) { w1 = nxt; }
		q0 = q1;
		q1 = q2;
		q2 = q3;
		q3 = ldw(ck + 4);
		const uint32_t b4    = off ? __funnelshift_r(w0, w1, 8u * off) : w0; // stream bytes cb+4l .. +3
		const uint32_t bnext = (w1 >> (8u * off)) & 0xFFu;                   // stream byte cb+4l+4
		const uint32_t pos0  = cb + 4 * lane;
		const uint32_t nv    = pos0 >= L ? 0u : (L - pos0 < 4u ? L - pos0 : 4u);
		uint64_t       sv[4];
		uint32_t       sl[4];
		if constexpr (!KIND_FSST) {
#pragma unroll
			for (uint32_t j = 0; j < 4; ++j) {
				sv[j] = j < nv ? (b4 >> (8 * j)) & 0xFFu : 0u;
				sl[j] = j < nv ? 1u : 0u;
			}
		} else {
			uint32_t esc = 0;
#pragma unroll
			for (uint32_t j = 0; j < 4; ++j) { esc |= (j < nv && ((b4 >> (8 * j)) & 0xFFu) == 255u) ? 1u << j : 0u; }
			if (!__any_sync(0xFFFFFFFFu, esc != 0 || carry != 0)) {
				// no escape anywhere in the chunk: every byte starts a code
#pragma unroll
				for (uint32_t j = 0; j < 4; ++j) {
					// a byte past the stream's end reads as code 255, whose table entry is empty (symbol 0, length 0)
					const uint32_t c = j < nv ? (b4 >> (8 * j)) & 0xFFu : 255u;
					sv[j]            = sym[c];
					sl[j]            = len[c];
				}
			} else {
				uint32_t m[4];
				bool     at_end;
				uint32_t r = rc;
				stream_row_mask(rows32, cb, lane, &r, m, &at_end);
				if constexpr (!MAT) { rc = r; }
				const uint32_t mk = (lane >> 3) == 0 ? m[0] : (lane >> 3) == 1 ? m[1] : (lane >> 3) == 2 ? m[2] : m[3];
				const uint32_t rs = (mk >> ((4 * lane) & 31u)) & 0xFu;
				uint32_t       rs4;
				if ((lane & 7u) != 7u) {
					rs4 = (mk >> ((4 * lane + 4) & 31u)) & 1u;
				} else {
					const uint32_t mn = (lane >> 3) == 0 ? m[1] : (lane >> 3) == 1 ? m[2] : m[3];
					rs4               = lane == 31 ? (at_end ? 1u : 0u) : (mn & 1u);
				}
				// entry state of every lane: warp scan of the transfer functions
				const uint32_t f    = esc_transfer(0, esc, rs, nv) | (esc_transfer(1, esc, rs, nv) << 1);
				uint32_t       incl = f;
#pragma unroll
				for (int d = 1; d < 32; d <<= 1) {
					const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
					if (lane >= static_cast<uint32_t>(d)) { incl = fn_compose(incl, y); }
				}
				uint32_t excl = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
				if (lane == 0) { excl = 2u; } // identity
				uint32_t       st  = fn_apply(excl, carry);
				const uint32_t all = __shfl_sync(0xFFFFFFFFu, incl, 31);
				carry              = fn_apply(all, carry);
#pragma unroll
				for (uint32_t j = 0; j < 4; ++j) {
					const uint32_t c = (b4 >> (8 * j)) & 0xFFu;
					sv[j]            = 0;
					sl[j]            = 0;
					if (j < nv) {
						if ((rs >> j) & 1u) { st = 0; }
						if (st) {
							st = 0; // the escaped literal: emitted with its escape
						} else if (c == 255u) {
							// the literal: the next byte unless the row (or the stream) ends first
							const uint32_t nb    = j < 3 ? (b4 >> (8 * (j + 1))) & 0xFFu : bnext;
							const bool     nvld  = j < 3 ? j + 1 < nv : pos0 + 4 < L;
							const bool     nrow  = j < 3 ? ((rs >> (j + 1)) & 1u) != 0 : rs4 != 0;
							sv[j]                = (nvld && !nrow) ? nb : 0u;
							sl[j]                = 1;
							st                   = 1;
						} else {
							sv[j] = sym[c];
							sl[j] = len[c];
						}
					}
				}
			}
		}
		// decoded offsets: lane sum, warp exclusive scan, chunk total
		const uint32_t e   = sl[0] + sl[1] + sl[2] + sl[3];
		const uint32_t inc = warp_inclusive_scan(e, lane);
		const uint32_t X   = inc - e;
		const uint32_t T   = __shfl_sync(0xFFFFFFFFu, inc, 31);
		if constexpr (MAT) {
			// offsets of the rows starting in this chunk (before cb + 128): from the owner lane of their first byte
			const uint32_t part = sl[0] | ((sl[0] + sl[1]) << 8) | ((sl[0] + sl[1] + sl[2]) << 16);
			while (rc < kVec) {
				const uint32_t rr  = rc + lane;
				const uint32_t s   = rr < kVec ? stream_row_start(rows32, rr) : 0xFFFFFFFFu;
				const bool     in  = s < cb + kStreamChunk;
				const uint32_t rel = s - cb;
				const uint32_t own = (rel >> 2) & 31u, sub = rel & 3u;
				const uint32_t xo  = __shfl_sync(0xFFFFFFFFu, X, own);
				const uint32_t po  = __shfl_sync(0xFFFFFFFFu, part, own);
				if (in) { o.offsets[rr] = static_cast<uint32_t>(o.vbase + vdec + xo + (sub ? (po >> (8 * (sub - 1))) & 0xFFu : 0u)); }
				const uint32_t n = __popc(__ballot_sync(0xFFFFFFFFu, in));
				rc += n;
				if (n < 32) { break; }
			}
			if (fill + T > kWindow) { flush(false); }
			uint32_t hk = 0, head = 0;
			const bool mid = put_syms(win32, fill + X, sv, sl, &hk, &head);
			__syncwarp(); // every word's whole store lands before the lanes that start inside it OR in
			if (mid) { atomicOr(win32 + hk, head); }
			__syncwarp();
			fill += T;
		}
		vdec += T;
	}
	if constexpr (MAT) {
		// rows starting at the stream's end (and every row of an empty or bad vector)
		for (uint32_t r = rc + lane; r < kVec; r += 32) { o.offsets[r] = static_cast<uint32_t>(o.vbase + vdec); }
		flush(true);
	}
	return vdec;
}

} // namespace flsgpu
