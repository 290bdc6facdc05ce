// Launchers, per-device runtime state and the C ABI of the primitive entry points (include/fls_b200.h).
#include "fls_b200.h"
#include "fls_decode.cu"
#include "fls_runtime.h"

#include <algorithm>
#include <cstdio>
#include <memory>
#include <mutex>
#include <vector>

namespace flsgpu {

// ---------------------------------------------------------------------------------------------------------
// Kernel families
// ---------------------------------------------------------------------------------------------------------
// <max stream width, run-value staging bytes, max output bytes, warps per CTA, staging depth, item kinds>
#define FLS_NUM64 64, 0u, 8, 12, 2, KIND_PLAIN
#define FLS_NUM32 32, 0u, 4, 15, 3, KIND_PLAIN
#define FLS_NUMPATCH 64, 0u, 8, 12, 2, KIND_PATCH
#define FLS_GATHER 32, 0u, 8, 10, 2, KIND_GATHER
#define FLS_GATHER32 32, 0u, 4, 12, 2, KIND_GATHER
#define FLS_ANY 64, 8320u, 8, 6, 2, KIND_ALL

template <int MAXWS, uint32_t GSTAGE, int EMAX, int WARPS, int STAGES, int KIND>
static cudaError_t launch_family(const DecodeArgs& a, cudaStream_t s, int sm_count, int grid_override) {
	using G            = Geometry<MAXWS, GSTAGE, EMAX, WARPS, STAGES, KIND>;
	auto*       kfn    = k_decode<MAXWS, GSTAGE, EMAX, WARPS, STAGES, KIND>;
	// per device: the shared-memory attribute is set and the occupancy queried once
	static int        occupancy[64] {};
	static std::mutex mu;
	int               dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { return cudaErrorInvalidDevice; }
	int per_sm = occupancy[dev];
	if (per_sm == 0) {
		std::lock_guard<std::mutex> lk(mu);
		cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
		if (e != cudaSuccess) { return e; }
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, G::kThreads, G::kSmem);
		if (e != cudaSuccess) { return e; }
		per_sm          = per_sm < 1 ? 1 : per_sm;
		occupancy[dev] = per_sm;
	}
	const uint64_t want = (a.n_items + WARPS - 1) / WARPS;
	uint64_t       grid = static_cast<uint64_t>(sm_count) * per_sm;
	if (grid_override > 0) { grid = static_cast<uint64_t>(grid_override); }
	if (want < grid) { grid = want; }
	if (grid == 0) { return cudaSuccess; }
	kfn<<<static_cast<unsigned>(grid), G::kThreads, G::kSmem, s>>>(a);
	++launch_counter();
	return cudaGetLastError();
}

uint64_t& launch_counter() {
	static uint64_t n = 0;
	return n;
}

// ---------------------------------------------------------------------------------------------------------
// Geometry variants of every family (warps per CTA x staging depth); variant 0 is the default, the others are
// what fls_plan_autotune chooses from on the plan's own data.
// ---------------------------------------------------------------------------------------------------------
struct Variant {
	const char* name;
	cudaError_t (*launch)(const DecodeArgs&, cudaStream_t, int, int);
	const void* kernel;
	int         threads, smem;
};

template <int MAXWS, uint32_t GSTAGE, int EMAX, int WARPS, int STAGES, int KIND>
static cudaError_t launch_variant(const DecodeArgs& a, cudaStream_t s, int sms, int grid) {
	return launch_family<MAXWS, GSTAGE, EMAX, WARPS, STAGES, KIND>(a, s, sms, grid);
}

#define FLS_VARIANT(label, ...)                                                                                   \
	Variant {                                                                                                     \
		label, launch_variant<__VA_ARGS__>, reinterpret_cast<const void*>(k_decode<__VA_ARGS__>),                 \
		    Geometry<__VA_ARGS__>::kThreads, static_cast<int>(Geometry<__VA_ARGS__>::kSmem)                       \
	}

static const Variant kNum64[]    = {FLS_VARIANT("num64 12x2", FLS_NUM64),
                                    FLS_VARIANT("num64 8x3", 64, 0u, 8, 8, 3, KIND_PLAIN),
                                    FLS_VARIANT("num64 10x2", 64, 0u, 8, 10, 2, KIND_PLAIN)};
static const Variant kNum32[]    = {FLS_VARIANT("num32 15x3", FLS_NUM32),
                                    FLS_VARIANT("num32 16x2", 32, 0u, 4, 16, 2, KIND_PLAIN),
                                    FLS_VARIANT("num32 10x4", 32, 0u, 4, 10, 4, KIND_PLAIN)};
static const Variant kNumPatch[] = {FLS_VARIANT("numpatch 12x2", FLS_NUMPATCH),
                                    FLS_VARIANT("numpatch 8x3", 64, 0u, 8, 8, 3, KIND_PATCH)};
static const Variant kGather[]   = {FLS_VARIANT("gather 10x2", FLS_GATHER),
                                    FLS_VARIANT("gather 8x3", 32, 0u, 8, 8, 3, KIND_GATHER),
                                    FLS_VARIANT("gather 12x2", 32, 0u, 8, 12, 2, KIND_GATHER)};
static const Variant kGather32[] = {FLS_VARIANT("gather32 12x2", FLS_GATHER32),
                                    FLS_VARIANT("gather32 12x3", 32, 0u, 4, 12, 3, KIND_GATHER),
                                    FLS_VARIANT("gather32 16x2", 32, 0u, 4, 16, 2, KIND_GATHER)};
static const Variant kAny[]      = {FLS_VARIANT("any 6x2", FLS_ANY)};
// filter launches (predicate bitmaps instead of values): the same geometries in their KIND_FILTER form
static const Variant kFNum64[]    = {FLS_VARIANT("filter num64 12x2", 64, 0u, 8, 12, 2, KIND_PLAIN | KIND_FILTER)};
static const Variant kFNum32[]    = {FLS_VARIANT("filter num32 15x3", 32, 0u, 4, 15, 3, KIND_PLAIN | KIND_FILTER)};
static const Variant kFNumPatch[] = {FLS_VARIANT("filter numpatch 12x2", 64, 0u, 8, 12, 2, KIND_PATCH | KIND_FILTER)};
static const Variant kFGather[]   = {FLS_VARIANT("filter gather 10x2", 32, 0u, 8, 10, 2, KIND_GATHER | KIND_FILTER)};
static const Variant kFGather32[] = {FLS_VARIANT("filter gather32 16x2", 32, 0u, 4, 16, 2, KIND_GATHER | KIND_FILTER)};
static const Variant kFAny[]      = {FLS_VARIANT("filter any 6x2", 64, 8320u, 8, 6, 2, KIND_ALL | KIND_FILTER)};

// The variants of a family; a NUM launch without a column array whose column is narrow runs the NUM32 kernels.
static const Variant* family_variants(Family fam, const DecodeArgs& a, int* n) {
	const bool narrow = a.cols == nullptr && a.col0.ws <= 32 && a.col0.e <= 4;
	if (a.pred.active) {
		*n = 1;
		switch (fam) {
		case Family::NUM_NARROW: return kFNum32;
		case Family::NUM: return narrow ? kFNum32 : kFNum64;
		case Family::NUM_PATCH: return kFNumPatch;
		case Family::GATHER: return kFGather;
		case Family::GATHER_NARROW: return kFGather32;
		default: return kFAny;
		}
	}
	auto count = [](const auto& arr) { return static_cast<int>(sizeof(arr) / sizeof(arr[0])); };
	switch (fam) {
	case Family::NUM_NARROW: *n = count(kNum32); return kNum32;
	case Family::NUM:
		*n = narrow ? count(kNum32) : count(kNum64);
		return narrow ? kNum32 : kNum64;
	case Family::NUM_PATCH: *n = count(kNumPatch); return kNumPatch;
	case Family::GATHER: *n = count(kGather); return kGather;
	case Family::GATHER_NARROW: *n = count(kGather32); return kGather32;
	default: *n = count(kAny); return kAny;
	}
}

int family_variant_count(Family fam, const DecodeArgs& a) {
	int n = 0;
	family_variants(fam, a, &n);
	return n;
}

const char* family_variant_name(Family fam, const DecodeArgs& a, int variant) {
	int            n = 0;
	const Variant* v = family_variants(fam, a, &n);
	return (variant >= 0 && variant < n) ? v[variant].name : "";
}

Device* current_device() {
	static Device     devs[64];
	static std::mutex mu;
	int               ord = 0;
	if (cudaGetDevice(&ord) != cudaSuccess || ord < 0 || ord >= 64) { return nullptr; }
	std::lock_guard<std::mutex> lk(mu);
	Device&                     d = devs[ord];
	if (d.ordinal < 0) {
		if (cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, ord) != cudaSuccess) { return nullptr; }
		if (cudaMalloc(&d.status, sizeof(int)) != cudaSuccess) { return nullptr; }
		if (cudaMemset(d.status, 0, sizeof(int)) != cudaSuccess) { return nullptr; }
		d.ordinal = ord;
	}
	return &d;
}

cudaError_t launch_decode(Family fam, const DecodeArgs& args, cudaStream_t stream, int grid_override, int variant) {
	Device* d = current_device();
	if (!d) { return cudaErrorInitializationError; }
	DecodeArgs a = args;
	if (!a.status) { a.status = d->status; }
	if (a.n_items == 0) { return cudaSuccess; }
	int            n = 0;
	const Variant* v = family_variants(fam, a, &n);
	if (variant < 0 || variant >= n) { variant = 0; }
	return v[variant].launch(a, stream, d->sm_count, grid_override);
}

void family_geometry(Family fam, const DecodeArgs& a, int variant, int* threads, int* smem, int* ctas_per_sm) {
	int            n = 0;
	const Variant* v = family_variants(fam, a, &n);
	if (variant < 0 || variant >= n) { variant = 0; }
	*threads = v[variant].threads;
	*smem    = v[variant].smem;
	int per  = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, v[variant].kernel, *threads, *smem);
	*ctas_per_sm = per;
}

// ---------------------------------------------------------------------------------------------------------
// Encoder-side kernels (fixtures, trial encodes, benchmark data).  Thread per lane of a vector.
// ---------------------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t transposed_index(uint32_t o) {
	// inverse of original_index: o = 64a + 8b + c  ->  k = a + 16*O[b] + 128*c   (O is an involution)
	return (o / 64) + 16 * fls_order((o / 8) % 8) + 128 * (o % 8);
}

template <typename T>
__global__ void k_permute(const T* __restrict__ in, T* __restrict__ out, uint64_t n_vec, bool to_transposed) {
	const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= n_vec * kVec) { return; }
	const uint64_t v = i / kVec;
	const uint32_t k = static_cast<uint32_t>(i % kVec);
	if (to_transposed) {
		out[i] = in[v * kVec + original_index(k)];
	} else {
		out[v * kVec + original_index(k)] = in[i];
	}
}

template <typename T, int W>
__global__ void k_ffor(const T* __restrict__ in, T* __restrict__ out, const uint8_t* __restrict__ bw,
                       const T* __restrict__ base, const uint64_t* __restrict__ byte_off, uint64_t n_vec) {
	// Word-centric packing: word w of lane l gathers every value j whose bits [j*b, (j+1)*b) overlap
	// [w*W, (w+1)*W).  Inverse of the unpack layout: lane l's word w lives at out[l + L*w].
	constexpr uint32_t L = 1024 / W;
	const uint64_t     i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= n_vec * L) { return; }
	const uint64_t v = i / L;
	const uint32_t l = static_cast<uint32_t>(i % L);
	const uint32_t b = bw[v];
	if (b == 0 || b > W) { return; }
	T* o = reinterpret_cast<T*>(reinterpret_cast<uint8_t*>(out) + (byte_off ? byte_off[v] : v * b * 128ull));
	const T        bs   = base ? base[v] : T(0);
	const T*       src  = in + v * kVec;
	const uint64_t mask = b >= 64 ? ~0ull : ((1ull << b) - 1ull);
	for (uint32_t w = 0; w < b; ++w) {
		const uint32_t lo_bit = w * W;
		const uint32_t j0     = lo_bit / b;
		const uint32_t j1     = (lo_bit + W - 1) / b;
		uint64_t       word   = 0;
		for (uint32_t j = j0; j <= j1 && j < static_cast<uint32_t>(W); ++j) {
			const uint64_t x  = static_cast<uint64_t>(static_cast<T>(src[l + L * j] - bs)) & mask;
			const int32_t  sh = static_cast<int32_t>(j * b) - static_cast<int32_t>(lo_bit);
			if (sh >= 0) {
				word |= sh >= 64 ? 0ull : (x << sh);
			} else {
				word |= (-sh) >= 64 ? 0ull : (x >> (-sh));
			}
		}
		o[l + L * w] = static_cast<T>(word);
	}
}

template <typename T, int W>
__global__ void k_unrsum(const T* __restrict__ in, T* __restrict__ out, uint64_t n_vec) {
	constexpr uint32_t L = 1024 / W;
	const uint64_t     i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= n_vec * L) { return; }
	const uint64_t v = i / L;
	const uint32_t l = static_cast<uint32_t>(i % L);
	// lane l covers a contiguous run of original positions; walk it in order
	uint32_t start;
	if constexpr (W == 64) {
		start = l * 64;
	} else if constexpr (W == 32) {
		start = (l % 16) * 64 + 32 * (l / 16);
	} else {
		start = (l % 16) * 64 + fls_order(l / 16) * 8;
	}
	const T* src  = in + v * kVec;
	T*       dst  = out + v * kVec;
	T        prev = 0;
	for (uint32_t p = 0; p < static_cast<uint32_t>(W); ++p) {
		const uint32_t k = transposed_index(start + p);
		const T        x = src[k];
		dst[k]           = p == 0 ? T(0) : static_cast<T>(x - prev);
		prev             = x;
	}
}

template <typename T, int W>
__global__ void k_analyze(const T* __restrict__ in, uint8_t* __restrict__ bw, T* __restrict__ base, uint64_t n_vec,
                          bool is_signed) {
	// one warp per vector
	const uint64_t v    = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
	const uint32_t lane = threadIdx.x & 31u;
	if (v >= n_vec) { return; }
	const T* src  = in + v * kVec;
	const T  flip = is_signed ? static_cast<T>(T(1) << (W - 1)) : T(0);
	T        mn = static_cast<T>(~T(0)), mx = 0;
	for (uint32_t k = lane; k < kVec; k += 32) {
		const T x = static_cast<T>(src[k] ^ flip);
		mn        = x < mn ? x : mn;
		mx        = x > mx ? x : mx;
	}
	for (int o = 16; o > 0; o >>= 1) {
		const T a = __shfl_xor_sync(0xFFFFFFFFu, mn, o);
		const T b = __shfl_xor_sync(0xFFFFFFFFu, mx, o);
		mn        = a < mn ? a : mn;
		mx        = b > mx ? b : mx;
	}
	if (lane == 0) {
		const uint64_t d = static_cast<uint64_t>(static_cast<T>(mx - mn));
		bw[v]            = static_cast<uint8_t>(d == 0 ? 0 : 64 - __clzll(static_cast<long long>(d)));
		base[v]          = static_cast<T>(mn ^ flip);
	}
}

} // namespace flsgpu

// =========================================================================================================
// C ABI
// =========================================================================================================
using namespace flsgpu;

namespace {
int to_status(cudaError_t e) { return e == cudaSuccess ? FLS_OK : FLS_ERR_CUDA; }

template <int W>
int run_primitive(const void* in, void* out, const uint8_t* bw, uint8_t bw_const, const void* base,
                  const void* lane_base, const uint64_t* byte_off, uint64_t n_vec, int order, uint8_t enc,
                  fls_stream_t stream) {
	if (n_vec == 0) { return FLS_OK; }
	if (!in || !out || (order != FLS_TRANSPOSED && order != FLS_ORIGINAL) || n_vec >= (1ull << 32)) {
		return FLS_ERR_ARG;
	}
	if ((reinterpret_cast<uintptr_t>(in) & 3u) != 0 || (reinterpret_cast<uintptr_t>(out) & (W / 8 - 1)) != 0) {
		return FLS_ERR_ARG;
	}
	if (bw_const > W) { return FLS_ERR_BW; }
	DecodeArgs a {};
	ColDesc&   c    = a.col0;
	c.ws            = W;
	c.e             = W / 8;
	c.enc           = enc;
	c.post          = POST_NONE;
	c.order         = static_cast<uint8_t>(order);
	c.layout        = LAYOUT_ARRAYS;
	c.n_vec         = static_cast<uint32_t>(n_vec);
	c.bw_const      = bw_const;
	c.packed        = static_cast<const uint8_t*>(in);
	c.byte_off      = byte_off;
	c.bw_arr        = bw;
	c.base_arr      = static_cast<const uint8_t*>(base);
	c.lane_base_arr = static_cast<const uint8_t*>(lane_base);
	c.out           = static_cast<uint8_t*>(out);
	a.n_items       = n_vec;
	return to_status(launch_decode(Family::NUM, a, static_cast<cudaStream_t>(stream)));
}

// The unffor primitive with failure injection (fls_gpu_test_stalled_copy).
int run_stalled(const uint32_t* in, uint32_t* out, const uint8_t* bw, const uint32_t* base, const uint64_t* byte_off,
                uint64_t n_vec, uint64_t stall_vector, uint32_t spin_limit, fls_stream_t stream) {
	if (!in || !out || !bw || !base || !byte_off || n_vec == 0 || n_vec >= (1ull << 32) || stall_vector >= n_vec ||
	    spin_limit == 0 || (reinterpret_cast<uintptr_t>(in) & 15u) != 0) {
		return FLS_ERR_ARG;
	}
	DecodeArgs a {};
	ColDesc&   c = a.col0;
	c.ws         = 32;
	c.e          = 4;
	c.enc        = ENC_FFOR;
	c.post       = POST_NONE;
	c.order      = FLS_TRANSPOSED;
	c.layout     = LAYOUT_ARRAYS;
	c.n_vec      = static_cast<uint32_t>(n_vec);
	c.packed     = reinterpret_cast<const uint8_t*>(in);
	c.byte_off   = byte_off;
	c.bw_arr     = bw;
	c.base_arr   = reinterpret_cast<const uint8_t*>(base);
	c.out        = reinterpret_cast<uint8_t*>(out);
	a.n_items    = n_vec;
	a.test_stall = stall_vector + 1;
	a.spin_limit = spin_limit;
	return to_status(launch_decode(Family::NUM, a, static_cast<cudaStream_t>(stream)));
}

template <typename T>
int run_permute(const T* in, T* out, uint64_t n_vec, bool to_transposed, fls_stream_t stream) {
	if (n_vec == 0) { return FLS_OK; }
	if (!in || !out) { return FLS_ERR_ARG; }
	const uint64_t n = n_vec * kVec;
	k_permute<T><<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, out, n_vec,
	                                                                                                    to_transposed);
	++launch_counter();
	return to_status(cudaGetLastError());
}

template <typename T, int W>
int run_ffor(const T* in, T* out, const uint8_t* bw, const T* base, const uint64_t* off, uint64_t n_vec,
             fls_stream_t stream) {
	if (n_vec == 0) { return FLS_OK; }
	if (!in || !out || !bw) { return FLS_ERR_ARG; }
	const uint64_t n = n_vec * (1024 / W);
	k_ffor<T, W><<<static_cast<unsigned>((n + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(in, out, bw,
	                                                                                                   base, off, n_vec);
	++launch_counter();
	return to_status(cudaGetLastError());
}

template <typename T, int W>
int run_unrsum(const T* in, T* out, uint64_t n_vec, fls_stream_t stream) {
	if (n_vec == 0) { return FLS_OK; }
	if (!in || !out || in == out) { return FLS_ERR_ARG; }
	const uint64_t n = n_vec * (1024 / W);
	k_unrsum<T, W><<<static_cast<unsigned>((n + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(in, out,
	                                                                                                     n_vec);
	++launch_counter();
	return to_status(cudaGetLastError());
}

template <typename T, int W>
int run_analyze(const T* in, uint8_t* bw, T* base, uint64_t n_vec, int is_signed, fls_stream_t stream) {
	if (n_vec == 0) { return FLS_OK; }
	if (!in || !bw || !base) { return FLS_ERR_ARG; }
	k_analyze<T, W><<<static_cast<unsigned>((n_vec + 7) / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
	    in, bw, base, n_vec, is_signed != 0);
	++launch_counter();
	return to_status(cudaGetLastError());
}
} // namespace

extern "C" {

int fls_gpu_status(int reset) {
	Device* d = current_device();
	if (!d) { return FLS_ERR_CUDA; }
	if (cudaDeviceSynchronize() != cudaSuccess) { return FLS_ERR_CUDA; }
	int h = 0;
	if (cudaMemcpy(&h, d->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) { return FLS_ERR_CUDA; }
	if (reset && cudaMemset(d->status, 0, sizeof(int)) != cudaSuccess) { return FLS_ERR_CUDA; }
	return h;
}

uint64_t fls_gpu_launch_count(int reset) {
	const uint64_t n = launch_counter();
	if (reset) { launch_counter() = 0; }
	return n;
}

int fls_gpu_test_stalled_copy(const uint32_t* d_in, uint32_t* d_out, const uint8_t* d_bw, const uint32_t* d_base,
                              const uint64_t* d_byte_off, uint64_t n_vec, uint64_t stall_vector, uint32_t spin_limit,
                              fls_stream_t stream) {
	return run_stalled(d_in, d_out, d_bw, d_base, d_byte_off, n_vec, stall_vector, spin_limit, stream);
}

#define FLS_PRIM(T, W)                                                                                                \
	int fls_gpu_unpack_u##W(const T* in, T* out, const uint8_t* bw, const uint64_t* off, uint64_t n, int order,     \
	                        fls_stream_t s) {                                                                       \
		if (!bw) { return FLS_ERR_ARG; }                                                                            \
		return run_primitive<W>(in, out, bw, 0, nullptr, nullptr, off, n, order, ENC_FFOR, s);                      \
	}                                                                                                               \
	int fls_gpu_unffor_u##W(const T* in, T* out, const uint8_t* bw, const T* base, const uint64_t* off, uint64_t n, \
	                        int order, fls_stream_t s) {                                                            \
		if (!bw || !base) { return FLS_ERR_ARG; }                                                                   \
		return run_primitive<W>(in, out, bw, 0, base, nullptr, off, n, order, ENC_FFOR, s);                         \
	}                                                                                                               \
	int fls_gpu_rsum_u##W(const T* in, T* out, const T* lane_base, uint64_t n, int order, fls_stream_t s) {         \
		if (!lane_base) { return FLS_ERR_ARG; }                                                                     \
		return run_primitive<W>(in, out, nullptr, W, nullptr, lane_base, nullptr, n, order, ENC_DELTA, s);          \
	}                                                                                                               \
	int fls_gpu_untranspose_i_u##W(const T* in, T* out, uint64_t n, fls_stream_t s) {                               \
		return run_primitive<W>(in, out, nullptr, W, nullptr, nullptr, nullptr, n, FLS_ORIGINAL, ENC_RAW, s);       \
	}                                                                                                               \
	int fls_gpu_transpose_i_u##W(const T* in, T* out, uint64_t n, fls_stream_t s) {                                 \
		return run_permute<T>(in, out, n, true, s);                                                                 \
	}                                                                                                               \
	int fls_gpu_ffor_u##W(const T* in, T* out, const uint8_t* bw, const T* base, const uint64_t* off, uint64_t n,   \
	                      fls_stream_t s) {                                                                         \
		return run_ffor<T, W>(in, out, bw, base, off, n, s);                                                        \
	}

FLS_PRIM(uint8_t, 8)
FLS_PRIM(uint16_t, 16)
FLS_PRIM(uint32_t, 32)
FLS_PRIM(uint64_t, 64)

#define FLS_PRIM2(T, W)                                                                                               \
	int fls_gpu_unffor_rsum_u##W(const T* in, T* out, const uint8_t* bw, const T* base, const T* lane_base,         \
	                             const uint64_t* off, uint64_t n, int order, fls_stream_t s) {                      \
		if (!bw || !base || !lane_base) { return FLS_ERR_ARG; }                                                     \
		return run_primitive<W>(in, out, bw, 0, base, lane_base, off, n, order, ENC_DELTA, s);                      \
	}                                                                                                               \
	int fls_gpu_unrsum_u##W(const T* in, T* out, uint64_t n, fls_stream_t s) { return run_unrsum<T, W>(in, out, n, s); } \
	int fls_gpu_analyze_u##W(const T* in, uint8_t* bw, T* base, uint64_t n, int sg, fls_stream_t s) {               \
		return run_analyze<T, W>(in, bw, base, n, sg, s);                                                           \
	}

FLS_PRIM2(uint16_t, 16)
FLS_PRIM2(uint32_t, 32)
FLS_PRIM2(uint64_t, 64)

} // extern "C"

// =========================================================================================================
// Plans
// =========================================================================================================
struct fls_plan {
	ColDesc*  d_cols   = nullptr;
	uint32_t* d_queue  = nullptr;
	uint64_t  n_items  = 0;
	uint32_t  n_cols   = 0;
	int       device   = -1;
	Family    family   = Family::NUM;
	uint32_t  col_shift = 24;
	ColDesc   col0 {};
	// launch segments: items [seg_begin[i], seg_begin[i + 1]) of the queue on family seg_fam[i]
	int       n_seg = 1;
	uint64_t  seg_begin[kMaxSegments + 1] {};
	Family    seg_fam[kMaxSegments] {};
	int       variant[kMaxSegments] {}; // geometry variant of each segment (fls_plan_autotune)
	std::vector<void*> owned;        // device buffers decoded for the plan (rec buffers)
	Pred               pred {};      // filter plans: the predicate of their FILTER launch
	cudaGraphExec_t graph = nullptr; // the segments' launches, captured by fls_plan_decode_graph
	cudaStream_t    graph_stream = nullptr;
};

namespace flsgpu {
void plan_adopt(::fls_plan* plan, std::vector<void*>&& buffers) {
	for (void* b : buffers) { plan->owned.push_back(b); }
}

void plan_set_filter(::fls_plan* plan, const Pred& pred) {
	// the plan's segments run the filter form of their families
	plan->pred        = pred;
	plan->pred.active = 1;
}

bool plan_segments(const std::vector<ColDesc>& descs, const std::vector<uint32_t>& queue, uint32_t col_shift,
                   Segments* out) {
	// a queue ordered by item class (plain streams, patched streams, gathers) decodes as one launch per class
	// present, each on the kernel specialised for it, instead of one launch of the catch-all kernel
	auto col   = [&](uint32_t it) -> const ColDesc& { return descs.size() == 1 ? descs[0] : descs[it >> col_shift]; };
	auto klass = [](const ColDesc& c) { return post_is_gather(c.post) ? 2 : post_is_patch(c.post) ? 1 : 0; };
	bool narrow[3] = {true, true, true};
	int  last      = -1;
	Segments s {};
	for (uint64_t i = 0; i < queue.size(); ++i) {
		const ColDesc& c = col(queue[i]);
		const int      k = klass(c);
		if (k < last) {
			*out         = Segments {};
			out->n       = 1;
			out->fam[0]  = Family::ANY;
			out->begin[1] = queue.size();
			return false;
		}
		if (k != last) {
			s.begin[s.n] = i;
			s.klass[s.n] = k;
			++s.n;
			last = k;
		}
		if (c.ws > 32 || c.e > 4) { narrow[k] = false; }
	}
	s.begin[s.n] = queue.size();
	for (int i = 0; i < s.n; ++i) {
		switch (s.klass[i]) {
		case 0: s.fam[i] = narrow[0] ? Family::NUM_NARROW : Family::NUM; break;
		case 1: s.fam[i] = Family::NUM_PATCH; break;
		default: s.fam[i] = narrow[2] ? Family::GATHER_NARROW : Family::GATHER; break;
		}
	}
	*out = s;
	return true;
}

int make_plan_object(const std::vector<ColDesc>& descs, const std::vector<uint32_t>& queue, Family fam,
                     uint32_t col_shift, ::fls_plan** out) {
	std::unique_ptr<fls_plan> p(new fls_plan());
	if (cudaGetDevice(&p->device) != cudaSuccess) { return FLS_ERR_CUDA; }
	p->n_cols    = static_cast<uint32_t>(descs.size());
	p->family    = fam;
	p->col_shift = col_shift;
	p->seg_fam[0]   = fam;
	p->seg_begin[1] = queue.size();
	if (!queue.empty()) {
		Segments sg;
		if (plan_segments(descs, queue, col_shift, &sg)) {
			p->n_seg = sg.n;
			for (int i = 0; i < sg.n; ++i) {
				p->seg_begin[i] = sg.begin[i];
				p->seg_fam[i]   = sg.fam[i];
			}
			p->seg_begin[sg.n] = sg.begin[sg.n];
		}
	}
	if (descs.size() == 1) {
		// one column: the queue is implicit (vector v = item v)
		p->col0    = descs[0];
		p->n_items = queue.size();
	} else {
		if (cudaMalloc(&p->d_cols, sizeof(ColDesc) * descs.size()) != cudaSuccess) { return FLS_ERR_CUDA; }
		if (cudaMemcpy(p->d_cols, descs.data(), sizeof(ColDesc) * descs.size(), cudaMemcpyHostToDevice) !=
		    cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		if (!queue.empty()) {
			if (cudaMalloc(&p->d_queue, sizeof(uint32_t) * queue.size()) != cudaSuccess) { return FLS_ERR_CUDA; }
			if (cudaMemcpy(p->d_queue, queue.data(), sizeof(uint32_t) * queue.size(), cudaMemcpyHostToDevice) !=
			    cudaSuccess) {
				return FLS_ERR_CUDA;
			}
		}
		p->n_items = queue.size();
	}
	*out = p.release();
	return FLS_OK;
}
} // namespace flsgpu

extern "C" {

int fls_plan_create(const fls_vector_batch* batches, uint32_t n_batches, const uint32_t* d_queue, uint64_t n_items,
                    fls_plan** out_plan) {
	return fls_plan_create_ex(batches, n_batches, d_queue, n_items, 0u, out_plan);
}

int fls_plan_create_ex(const fls_vector_batch* batches, uint32_t n_batches, const uint32_t* d_queue, uint64_t n_items,
                       uint32_t flags, fls_plan** out_plan) {
	if (!out_plan || !batches || n_batches == 0 || n_batches > 256) { return FLS_ERR_ARG; }
	*out_plan = nullptr;
	std::unique_ptr<fls_plan> p(new fls_plan());
	std::vector<ColDesc>     cols(n_batches);
	uint64_t                 total = 0;
	for (uint32_t i = 0; i < n_batches; ++i) {
		const fls_vector_batch& b = batches[i];
		if (b.width != 8 && b.width != 16 && b.width != 32 && b.width != 64) { return FLS_ERR_ARG; }
		if (b.encoding > FLS_ENC_DELTA || b.order > FLS_ORIGINAL || !b.d_packed || !b.d_out) { return FLS_ERR_ARG; }
		if (b.encoding != FLS_ENC_RAW && (!b.d_bw || !b.d_base || !b.d_byte_off)) { return FLS_ERR_ARG; }
		if (b.encoding == FLS_ENC_DELTA && !b.d_lane_base) { return FLS_ERR_ARG; }
		if (b.n_vec >= (1u << 24)) { return FLS_ERR_ARG; }
		ColDesc& c      = cols[i];
		c               = ColDesc {};
		c.ws            = b.width;
		c.e             = b.width / 8;
		c.enc           = b.encoding;
		c.post          = POST_NONE;
		c.order         = b.order;
		c.layout        = LAYOUT_ARRAYS;
		c.n_vec         = b.n_vec;
		c.bw_const      = b.encoding == FLS_ENC_RAW ? b.width : 0;
		c.packed        = static_cast<const uint8_t*>(b.d_packed);
		c.byte_off      = b.encoding == FLS_ENC_RAW ? nullptr : b.d_byte_off;
		c.bw_arr        = b.encoding == FLS_ENC_RAW ? nullptr : b.d_bw;
		c.base_arr      = static_cast<const uint8_t*>(b.d_base);
		c.lane_base_arr = static_cast<const uint8_t*>(b.d_lane_base);
		c.out           = static_cast<uint8_t*>(b.d_out);
		total += b.n_vec;
	}
	if (cudaGetDevice(&p->device) != cudaSuccess) { return FLS_ERR_CUDA; }
	p->n_cols = n_batches;
	p->family = Family::NUM;
	if (n_batches == 1 && d_queue == nullptr) {
		p->col0    = cols[0];
		p->n_items = total;
	} else {
		std::vector<uint32_t> q;
		if (d_queue == nullptr) {
			q.reserve(total);
			for (uint32_t i = 0; i < n_batches; ++i) {
				for (uint32_t v = 0; v < cols[i].n_vec; ++v) { q.push_back((i << 24) | v); }
			}
			n_items = total;
		} else {
			q.resize(n_items);
			if (n_items && cudaMemcpy(q.data(), d_queue, sizeof(uint32_t) * n_items, cudaMemcpyDeviceToHost) !=
			                   cudaSuccess) {
				return FLS_ERR_CUDA;
			}
		}
		for (uint32_t it : q) {
			if ((it >> 24) >= n_batches || (it & 0xFFFFFFu) >= cols[it >> 24].n_vec) { return FLS_ERR_ARG; }
		}
		if (!(flags & FLS_PLAN_KEEP_ORDER)) {
			// Group the work items by kernel specialisation (stream width, output size, encoding, order) so
			// that the warps of the persistent kernel run long stretches of one code path; within a group the
			// queue order is kept.  Outputs do not depend on the order.
			auto key = [&](uint32_t it) {
				const ColDesc& c = cols[it >> 24];
				return (c.ws << 24) | (c.e << 16) | (c.enc << 8) | (c.post << 4) | c.order;
			};
			std::stable_sort(q.begin(), q.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
		}
		if (cudaMalloc(&p->d_cols, sizeof(ColDesc) * n_batches) != cudaSuccess) { return FLS_ERR_CUDA; }
		if (cudaMemcpy(p->d_cols, cols.data(), sizeof(ColDesc) * n_batches, cudaMemcpyHostToDevice) != cudaSuccess) {
			return FLS_ERR_CUDA;
		}
		if (n_items > 0) {
			if (cudaMalloc(&p->d_queue, sizeof(uint32_t) * n_items) != cudaSuccess) { return FLS_ERR_CUDA; }
			const cudaError_t e =
			    cudaMemcpy(p->d_queue, q.data(), sizeof(uint32_t) * n_items, cudaMemcpyHostToDevice);
			if (e != cudaSuccess) { return FLS_ERR_CUDA; }
		}
		p->n_items = n_items;
	}
	*out_plan = p.release();
	return FLS_OK;
}

namespace {

// The launch arguments of segment `seg` (0 or 1) of a plan; false when the plan has no such segment.
bool segment_args(const fls_plan* p, int seg, DecodeArgs* a, Family* fam) {
	if (seg < 0 || seg >= p->n_seg) { return false; }
	DecodeArgs x {};
	x.cols      = p->d_cols;
	x.queue     = p->d_queue ? p->d_queue + p->seg_begin[seg] : nullptr;
	x.col_shift = p->col_shift;
	x.col0      = p->col0;
	x.n_items   = p->n_seg == 1 ? p->n_items : p->seg_begin[seg + 1] - p->seg_begin[seg];
	x.pred      = p->pred;
	*fam        = p->seg_fam[seg];
	*a          = x;
	return true;
}

int launch_segments(const fls_plan* p, int grid, cudaStream_t s) {
	for (int seg = 0; seg < p->n_seg; ++seg) {
		DecodeArgs a;
		Family     fam;
		if (!segment_args(p, seg, &a, &fam)) { break; }
		const int rc = to_status(launch_decode(fam, a, s, grid, p->variant[seg]));
		if (rc != FLS_OK) { return rc; }
	}
	return FLS_OK;
}

void drop_graph(fls_plan* p) {
	if (p->graph) {
		cudaGraphExecDestroy(p->graph);
		p->graph = nullptr;
	}
}

} // namespace

int fls_plan_decode_grid(const fls_plan* p, int grid, fls_stream_t stream) {
	if (!p) { return FLS_ERR_ARG; }
	return launch_segments(p, grid, static_cast<cudaStream_t>(stream));
}

int fls_plan_decode(const fls_plan* p, fls_stream_t stream) { return fls_plan_decode_grid(p, 0, stream); }

int fls_plan_decode_graph(fls_plan* p, fls_stream_t stream) {
	if (!p) { return FLS_ERR_ARG; }
	if (!p->graph) {
		// capture on a private stream (the legacy default stream cannot be captured); relaxed mode, since the
		// first launch of a kernel family sets its shared-memory attribute
		cudaStream_t cs = nullptr;
		if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { return FLS_ERR_CUDA; }
		cudaGraph_t g  = nullptr;
		int         rc = FLS_OK;
		if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
			rc = FLS_ERR_CUDA;
		} else {
			const uint64_t launches = launch_counter();
			rc                      = launch_segments(p, 0, cs);
			launch_counter()        = launches;
			if (cudaStreamEndCapture(cs, &g) != cudaSuccess && rc == FLS_OK) { rc = FLS_ERR_CUDA; }
		}
		if (rc == FLS_OK && (!g || cudaGraphInstantiate(&p->graph, g, 0) != cudaSuccess)) { rc = FLS_ERR_CUDA; }
		if (g) { cudaGraphDestroy(g); }
		cudaStreamDestroy(cs);
		if (rc != FLS_OK) { return rc; }
	}
	if (cudaGraphLaunch(p->graph, static_cast<cudaStream_t>(stream)) != cudaSuccess) { return FLS_ERR_CUDA; }
	launch_counter() += static_cast<uint64_t>(p->n_seg);
	return FLS_OK;
}

int fls_plan_autotune(fls_plan* p, int reps, fls_stream_t stream) {
	if (!p || reps < 1) { return FLS_ERR_ARG; }
	cudaStream_t s  = static_cast<cudaStream_t>(stream);
	cudaEvent_t  e0 = nullptr, e1 = nullptr;
	if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) { return FLS_ERR_CUDA; }
	int rc = FLS_OK;
	for (int seg = 0; seg < p->n_seg && rc == FLS_OK; ++seg) {
		DecodeArgs a;
		Family     fam;
		if (!segment_args(p, seg, &a, &fam)) { break; }
		const int n    = family_variant_count(fam, a);
		float     best = 0.0f;
		int       pick = 0;
		for (int v = 0; v < n && rc == FLS_OK; ++v) {
			// one untimed launch (first use sets the kernel's attributes), then `reps` timed ones
			rc = to_status(launch_decode(fam, a, s, 0, v));
			if (rc != FLS_OK) { break; }
			cudaEventRecord(e0, s);
			for (int r = 0; r < reps && rc == FLS_OK; ++r) { rc = to_status(launch_decode(fam, a, s, 0, v)); }
			cudaEventRecord(e1, s);
			float ms = 0.0f;
			if (rc == FLS_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)) {
				rc = FLS_ERR_CUDA;
			}
			if (rc == FLS_OK && (v == 0 || ms < best)) {
				best = ms;
				pick = v;
			}
		}
		p->variant[seg] = pick;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	drop_graph(p);
	return rc;
}

const char* fls_plan_variant_name(const fls_plan* p, int segment) {
	if (!p || segment < 0 || segment >= kMaxSegments) { return ""; }
	DecodeArgs a;
	Family     fam;
	if (!segment_args(p, segment, &a, &fam)) { return ""; }
	return family_variant_name(fam, a, p->variant[segment]);
}

int fls_plan_destroy(fls_plan* p) {
	if (!p) { return FLS_OK; }
	drop_graph(p);
	for (void* b : p->owned) { cudaFree(b); }
	if (p->d_cols) { cudaFree(p->d_cols); }
	if (p->d_queue) { cudaFree(p->d_queue); }
	delete p;
	return FLS_OK;
}

int fls_plan_geometry(const fls_plan* p, int* threads, int* smem_bytes, int* ctas_per_sm) {
	if (!p || !threads || !smem_bytes || !ctas_per_sm) { return FLS_ERR_ARG; }
	DecodeArgs a {};
	Family     fam = Family::NUM;
	segment_args(p, 0, &a, &fam);
	family_geometry(fam, a, p->variant[0], threads, smem_bytes, ctas_per_sm);
	return FLS_OK;
}

} // extern "C"
