// Internal runtime interface between the C++ host code (page walking, column API) and the CUDA launchers.
#pragma once

#include "fls_plan.h"
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

struct fls_plan; // the opaque plan of include/fls_b200.h

namespace flsgpu {

enum class Family : int {
	NUM        = 0, // streams up to 64 bits, no gather (FFOR / DELTA / raw, incl. primitive API)
	GATHER     = 1, // streams up to 32 bits with RLE run values staged and/or a dictionary gather, outputs up to 8 B
	ANY           = 2, // everything
	NUM_NARROW    = 3, // NUM with every stream and output at most 32 bits
	GATHER_NARROW = 4, // GATHER with outputs of at most 4 bytes
	NUM_PATCH     = 5, // NUM items with patches (S / B / LL) applied before rsum
};

// Launch segments of a queue ordered by item class (plain, patched, gather): at most one per class.
constexpr int kMaxSegments = 3;
struct Segments {
	int      n = 0;
	uint64_t begin[kMaxSegments + 1] {};
	int      klass[kMaxSegments] {};
	Family   fam[kMaxSegments] {};
};

// Per-device state: SM count and the library-owned status word.
struct Device {
	int  ordinal  = -1;
	int  sm_count = 0;
	int* status   = nullptr; // cudaMalloc'd once, 4 bytes
};

// Returns the state of the current device (initialising it on first use), or nullptr on a CUDA error.
Device* current_device();

// Launch the persistent decode kernel of the given family in geometry variant `variant` (0 = the default;
// grid_override 0 = one wave of resident CTAs).
cudaError_t launch_decode(Family fam, const DecodeArgs& args, cudaStream_t stream, int grid_override = 0,
                          int variant = 0);
int         family_variant_count(Family fam, const DecodeArgs& args);
const char* family_variant_name(Family fam, const DecodeArgs& args, int variant);

// Geometry of a family variant for these launch arguments (threads per CTA, dynamic shared memory per CTA,
// CTAs resident per SM).
void family_geometry(Family fam, const DecodeArgs& args, int variant, int* threads, int* smem, int* ctas_per_sm);

// Kernel families for a queue of (col << col_shift | vec) items ordered by class (plain streams, patched
// streams, gathers): one segment per class present.  Returns false (one ANY segment) for an unordered queue.
bool plan_segments(const std::vector<ColDesc>& descs, const std::vector<uint32_t>& queue, uint32_t col_shift,
                   Segments* out);

// Build a plan object from descriptors + queue of (col << col_shift | vec) items (uploads both; a single column
// without a queue stays inline).
int make_plan_object(const std::vector<ColDesc>& descs, const std::vector<uint32_t>& queue, Family fam,
                     uint32_t col_shift, ::fls_plan** out);

// Hand device buffers to a plan: freed when the plan is destroyed.
void plan_adopt(::fls_plan* plan, std::vector<void*>&& buffers);
// Turn a page plan into a filter plan: its launches evaluate `pred` with the KIND_FILTER form of each segment's
// kernel family (its columns' descriptors carry OUT_BITMAP_* and bitmap outputs).
void plan_set_filter(::fls_plan* plan, const Pred& pred);

// Kernels launched by this library inside the last timed region of a caller (a plain counter; not thread-safe).
uint64_t& launch_counter();

} // namespace flsgpu
