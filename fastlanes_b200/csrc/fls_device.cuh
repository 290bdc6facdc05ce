// Device building blocks of the B200 FastLanes decode engine (sm_100a).
//
// One warp owns one 1024-value vector in the FastLanes unified transposed layout:
//     transposed[k] = original[(k % 16) * 64 + O[(k / 16) % 8] * 8 + k / 128],  O = {0,4,2,6,1,5,3,7}
// (the permutation of primitives/fls_generated/fallback/scalar_aav_uf1/*_transpose_src.cpp, identical for
// every type width).  A W-bit stream has L = 1024/W lanes; lane i's packed word w is in[i + L*w] and lane
// i's value j lives at transposed position i + L*j.  Since a row of L words is always 128 bytes, the warp
// reads packed data as 32-bit words S[t + 32*w], which puts every thread on its own shared-memory bank:
//   W = 32: thread t owns lane t (32 values)
//   W = 64: thread t owns half t/16 of lane t%16 (the 32 odd or even values of that lane)
//   W = 16: thread t owns lanes 2t, 2t+1 (16 values each; both halves of S[t + 32*w])
//   W =  8: thread t owns lanes 4t..4t+3 (8 values each; the bytes of S[t + 32*w])
// In every case a thread's 32 values are contiguous runs of the ORIGINAL order, which makes delta decoding
// (the reference's rsum) a register scan and untransposing a question of where the runs are written.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace flsgpu {

constexpr uint32_t kVec = 1024;

#ifndef FLS_HOST_EMULATION // the tests compile the pure device logic below as host code; PTX stays here

// ---------------------------------------------------------------------------------------------------------
// PTX wrappers: mbarrier + bulk (non-tensor) TMA copies global -> shared.  No multicast anywhere.
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
	             : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	                 smem_addr(dst)),
	             "l"(src), "r"(bytes), "r"(smem_addr(bar))
	             : "memory");
}

// Bulk prefetch of a global range into L2 (no completion, no shared memory); 16-byte aligned start and size.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
	asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}\n"
	    : "=r"(ok)
	    : "r"(smem_addr(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}

// Bounded wait: every spin in this library ends.  try_wait itself suspends for a hardware-defined interval,
// so the bound below is far beyond any legitimate copy latency.
constexpr uint32_t kMbarSpinLimit = 1u << 20;

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kMbarSpinLimit) {
	for (uint32_t i = 0; i < limit; ++i) {
		if (mbar_try_wait(bar, parity)) { return true; }
	}
	return false;
}

#endif // FLS_HOST_EMULATION

// ---------------------------------------------------------------------------------------------------------
// Layout helpers
// ---------------------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t fls_order(uint32_t i) {
	// O = {0,4,2,6,1,5,3,7} packed as nibbles
	return (0x73516240u >> (4 * i)) & 7u;
}

__host__ __device__ __forceinline__ uint32_t original_index(uint32_t k) {
	return (k % 16) * 64 + fls_order((k / 16) % 8) * 8 + k / 128;
}

// Position inside a 32-value run of value j (W = 32: lane value j; W = 64: half-lane value m).
// {0,2,1,3}[j % 4] * 8 + j / 4
__host__ __device__ constexpr uint32_t run32_pos(uint32_t j) {
	return ((0x3120u >> (4 * (j % 4))) & 0xFu) * 8 + j / 4;
}
// Inverse of run32_pos: which value j lands at run position p.
__host__ __device__ constexpr uint32_t run32_val(uint32_t p) {
	return ((0x3120u >> (4 * (p / 8))) & 0xFu) + 4 * (p % 8);
}
// W = 16: position of lane value j inside its 16-value run, and the inverse.
__host__ __device__ constexpr uint32_t run16_pos(uint32_t j) { return (j % 2) * 8 + j / 2; }
__host__ __device__ constexpr uint32_t run16_val(uint32_t p) { return (p % 8) * 2 + p / 8; }

// Swizzle of the original-order staging buffer: 16-byte chunk c of 128-byte row r lives at chunk
// c ^ swz(r).  Chosen so that the run writes of every stream width and the row-wise read-back are free of
// shared-memory bank conflicts.
__device__ __forceinline__ uint32_t swz(uint32_t row) { return (row ^ (row >> 3)) & 7u; }

__device__ __forceinline__ uint32_t stage_off(uint32_t byte_off) {
	const uint32_t row = byte_off >> 7;
	return (row << 7) | ((((byte_off >> 4) & 7u) ^ swz(row)) << 4) | (byte_off & 15u);
}

template <int W>
struct UT;
template <>
struct UT<8> {
	using T = uint8_t;
};
template <>
struct UT<16> {
	using T = uint16_t;
};
template <>
struct UT<32> {
	using T = uint32_t;
};
template <>
struct UT<64> {
	using T = uint64_t;
};

// ---------------------------------------------------------------------------------------------------------
// Bit extraction: S = staged packed words of one vector (bw rows of 128 bytes; one further row of any
// readable shared memory must follow, its contents are masked off).
// v[i] receives this thread's values in RUN order (see the header comment): the permutation from lane
// value index to run position is a compile-time register renaming.
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void extract_w32(const uint32_t* __restrict__ S, uint32_t t, uint32_t bw,
                                            uint32_t (&v)[32]) {
	const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
#pragma unroll
	for (uint32_t j = 0; j < 32; ++j) {
		const uint32_t b  = j * bw;
		const uint32_t w  = b >> 5;
		const uint32_t lo = S[t + 32 * w];
		const uint32_t hi = S[t + 32 * w + 32];
		v[run32_pos(j)]   = __funnelshift_r(lo, hi, b & 31u) & mask;
	}
}

__device__ __forceinline__ void extract_w64(const uint32_t* __restrict__ S, uint32_t t, uint32_t bw,
                                            uint64_t (&v)[32]) {
	const uint32_t l     = t & 15u;
	const uint32_t h     = t >> 4;
	const uint64_t mask  = bw >= 64 ? ~0ull : ((1ull << bw) - 1ull);
	const uint32_t mlo   = static_cast<uint32_t>(mask);
	const uint32_t mhi   = static_cast<uint32_t>(mask >> 32);
	const uint2*   S2    = reinterpret_cast<const uint2*>(S);
	if (bw <= 32) {
		// a value of at most 32 bits lies in two adjacent 32-bit halves of the lane's 64-bit words: half-word
		// index 2w (+1 when s >= 32) of word w = b >> 6, i.e. half h2 = b >> 5 of the lane
#pragma unroll
		for (uint32_t m = 0; m < 32; ++m) {
			const uint32_t j  = 2 * m + h;
			const uint32_t b  = j * bw;
			const uint32_t h2 = b >> 5;
			const uint32_t lo = S[2 * (l + 16 * (h2 >> 1)) + (h2 & 1u)];
			const uint32_t h3 = h2 + 1;
			const uint32_t hi = S[2 * (l + 16 * (h3 >> 1)) + (h3 & 1u)];
			v[run32_pos(m)]   = __funnelshift_r(lo, hi, b & 31u) & mlo;
		}
		return;
	}
#pragma unroll
	for (uint32_t m = 0; m < 32; ++m) {
		const uint32_t j   = 2 * m + h;
		const uint32_t b   = j * bw;
		const uint32_t w   = b >> 6;
		const uint32_t s   = b & 63u;
		const uint2    lo  = S2[l + 16 * w];
		const uint2    hi  = S2[l + 16 * w + 16];
		const bool     up  = s >= 32;
		const uint32_t a   = up ? lo.y : lo.x;
		const uint32_t bb  = up ? hi.x : lo.y;
		const uint32_t c   = up ? hi.y : hi.x;
		const uint32_t sh  = s & 31u;
		const uint32_t xlo = __funnelshift_r(a, bb, sh) & mlo;
		const uint32_t xhi = __funnelshift_r(bb, c, sh) & mhi;
		v[run32_pos(m)]    = (static_cast<uint64_t>(xhi) << 32) | xlo;
	}
}

// W = 16: v[16*q + p] is run position p of lane 2t+q.
__device__ __forceinline__ void extract_w16(const uint32_t* __restrict__ S, uint32_t t, uint32_t bw,
                                            uint32_t (&v)[32]) {
	if (bw <= 1) {
		// every value of the thread's two lanes is one bit of its first packed word (RLE run-index deltas
		// are 0 or 1, so every RLE and DICT_RLE vector takes this path)
		const uint32_t lo = bw ? S[t] : 0u;
#pragma unroll
		for (uint32_t j = 0; j < 16; ++j) {
			v[run16_pos(j)]      = (lo >> j) & 1u;
			v[16 + run16_pos(j)] = (lo >> (16 + j)) & 1u;
		}
		return;
	}
	const uint32_t mask = bw >= 16 ? 0xFFFFu : ((1u << bw) - 1u);
#pragma unroll
	for (uint32_t j = 0; j < 16; ++j) {
		const uint32_t b       = j * bw;
		const uint32_t w       = b >> 4;
		const uint32_t s       = b & 15u;
		const uint32_t lo      = S[t + 32 * w];
		const uint32_t hi      = S[t + 32 * w + 32];
		v[run16_pos(j)]        = (__byte_perm(lo, hi, 0x5410) >> s) & mask;
		v[16 + run16_pos(j)]   = (__byte_perm(lo, hi, 0x7632) >> s) & mask;
	}
}

// W = 8: v[8*q + j] is value j (= run position j) of lane 4t+q.
__device__ __forceinline__ void extract_w8(const uint32_t* __restrict__ S, uint32_t t, uint32_t bw,
                                           uint32_t (&v)[32]) {
	const uint32_t mask = bw >= 8 ? 0xFFu : ((1u << bw) - 1u);
#pragma unroll
	for (uint32_t j = 0; j < 8; ++j) {
		const uint32_t b  = j * bw;
		const uint32_t w  = b >> 3;
		const uint32_t s  = b & 7u;
		const uint32_t lo = S[t + 32 * w];
		const uint32_t hi = S[t + 32 * w + 32];
#pragma unroll
		for (uint32_t q = 0; q < 4; ++q) {
			v[8 * q + j] = (__byte_perm(lo, hi, q | ((q + 4) << 4)) >> s) & mask;
		}
	}
}

// Original-order start (in values) of run r of thread t for stream width W, and the run length.
template <int W>
__device__ __forceinline__ uint32_t run_start(uint32_t t, uint32_t r) {
	if constexpr (W == 32) {
		return (t % 16) * 64 + 32 * (t / 16);
	} else if constexpr (W == 64) {
		return (t & 15u) * 64 + 32 * (t >> 4);
	} else if constexpr (W == 16) {
		const uint32_t l = 2 * t + r;
		return (l % 16) * 64 + fls_order(l / 16) * 8;
	} else {
		const uint32_t l = 4 * t + r;
		return (l % 16) * 64 + fls_order(l / 16) * 8;
	}
}
template <int W>
__host__ __device__ constexpr uint32_t run_len() {
	return W == 16 ? 16 : (W == 8 ? 8 : 32);
}
template <int W>
__host__ __device__ constexpr uint32_t run_count() {
	return 32 / run_len<W>();
}

// Transposed position of run position p of run r of thread t.
template <int W>
__device__ __forceinline__ uint32_t run_tpos(uint32_t t, uint32_t r, uint32_t p) {
	if constexpr (W == 32) {
		return t + 32 * run32_val(p);
	} else if constexpr (W == 64) {
		return (t & 15u) + 16 * (2 * run32_val(p) + (t >> 4));
	} else if constexpr (W == 16) {
		return 2 * t + r + 64 * run16_val(p);
	} else {
		return 4 * t + r + 128 * p;
	}
}

} // namespace flsgpu
