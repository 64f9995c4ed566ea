// Test-only link shim for the reference's cuda/memory.cu (cuda/memory.cu:6-21).
//
// The reference SBVH keeps its arrays in CUDA managed memory (ksc::CudaManagedArray,
// cuda/memory.cuh:557).  The oracle runs the reference builder and traversal on the host only,
// so the three allocation entry points are replaced by plain aligned host allocations.  This is
// what lets the unmodified builder run in a container with no GPU.
#include <cstddef>
#include <cstdlib>

namespace ksc
{
void *cuda_alloc_managed(size_t size) { return std::aligned_alloc(256, (size + 255) / 256 * 256); }
void *cuda_alloc_device(size_t size) { return std::aligned_alloc(256, (size + 255) / 256 * 256); }
void cuda_free(void *ptr) { std::free(ptr); }
} // namespace ksc
