// Stand-in for <cuda_runtime.h> when the decode engine's device logic is compiled as host code for the
// warp-emulation tests.  Defines the CUDA qualifiers away and emulates the warp intrinsics the decode
// functions use: a warp is 32 std::threads sharing a barrier.
#pragma once
#include <barrier>
#include <cstdint>
#include <cstring>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __align__(n) __attribute__((aligned(n)))
#define __restrict__ __restrict

typedef int           cudaError_t;
typedef struct CUst_* cudaStream_t;
#define cudaSuccess 0

struct uint2 {
	uint32_t x, y;
};
struct uint4 {
	uint32_t x, y, z, w;
};
inline uint4 make_uint4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return {a, b, c, d}; }
inline uint2 make_uint2(uint32_t a, uint32_t b) { return {a, b}; }

inline uint32_t __funnelshift_r(uint32_t lo, uint32_t hi, uint32_t s) {
	const uint64_t x = (static_cast<uint64_t>(hi) << 32) | lo;
	return static_cast<uint32_t>(x >> (s & 31u));
}
inline uint32_t __funnelshift_l(uint32_t lo, uint32_t hi, uint32_t s) {
	const uint64_t x = (static_cast<uint64_t>(hi) << 32) | lo;
	return static_cast<uint32_t>((x << (s & 31u)) >> 32);
}
inline uint32_t __byte_perm(uint32_t x, uint32_t y, uint32_t s) {
	uint8_t b[8];
	std::memcpy(b, &x, 4);
	std::memcpy(b + 4, &y, 4);
	uint32_t r = 0;
	for (int i = 0; i < 4; ++i) { r |= static_cast<uint32_t>(b[(s >> (4 * i)) & 7u]) << (8 * i); }
	return r;
}
inline int __clzll(long long x) { return x ? __builtin_clzll(static_cast<unsigned long long>(x)) : 64; }

struct EmuWarp {
	std::barrier<>* bar;
	uint64_t        xch[32];
	int             vote[32];
};
extern thread_local EmuWarp* g_emu_warp;
extern thread_local int      g_emu_lane;

inline void __syncwarp(unsigned = 0xFFFFFFFFu) { g_emu_warp->bar->arrive_and_wait(); }
template <class T>
T __shfl_sync(unsigned, T v, int src) {
	g_emu_warp->xch[g_emu_lane] = static_cast<uint64_t>(v);
	__syncwarp();
	const T r = static_cast<T>(g_emu_warp->xch[src & 31]);
	__syncwarp();
	return r;
}
template <class T>
T __shfl_up_sync(unsigned, T v, unsigned d) {
	g_emu_warp->xch[g_emu_lane] = static_cast<uint64_t>(v);
	__syncwarp();
	const T r = g_emu_lane >= static_cast<int>(d) ? static_cast<T>(g_emu_warp->xch[g_emu_lane - d]) : v;
	__syncwarp();
	return r;
}
template <class T>
T __shfl_down_sync(unsigned, T v, unsigned d) {
	g_emu_warp->xch[g_emu_lane] = static_cast<uint64_t>(v);
	__syncwarp();
	const T r = g_emu_lane + static_cast<int>(d) < 32 ? static_cast<T>(g_emu_warp->xch[g_emu_lane + d]) : v;
	__syncwarp();
	return r;
}
template <class T>
T __shfl_xor_sync(unsigned, T v, int m) {
	g_emu_warp->xch[g_emu_lane] = static_cast<uint64_t>(v);
	__syncwarp();
	const T r = static_cast<T>(g_emu_warp->xch[(g_emu_lane ^ m) & 31]);
	__syncwarp();
	return r;
}
inline unsigned __reduce_or_sync(unsigned, unsigned v) {
	g_emu_warp->xch[g_emu_lane] = v;
	__syncwarp();
	unsigned r = 0;
	for (int i = 0; i < 32; ++i) { r |= static_cast<unsigned>(g_emu_warp->xch[i]); }
	__syncwarp();
	return r;
}
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
inline bool __any_sync(unsigned, bool p) {
	g_emu_warp->vote[g_emu_lane] = p ? 1 : 0;
	__syncwarp();
	bool r = false;
	for (int i = 0; i < 32; ++i) { r = r || g_emu_warp->vote[i]; }
	__syncwarp();
	return r;
}
inline unsigned __ballot_sync(unsigned, bool p) {
	g_emu_warp->vote[g_emu_lane] = p ? 1 : 0;
	__syncwarp();
	unsigned r = 0;
	for (int i = 0; i < 32; ++i) { r |= (g_emu_warp->vote[i] ? 1u : 0u) << i; }
	__syncwarp();
	return r;
}
inline int atomicOr(int* a, int v) { return __atomic_fetch_or(a, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicOr(unsigned* a, unsigned v) { return __atomic_fetch_or(a, v, __ATOMIC_SEQ_CST); }
template <class T>
T __ldg(const T* p) {
	return *p;
}
