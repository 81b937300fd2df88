// Drop-in replacement for the reference's include/types.hpp.
//
// Same names and values for the SpMV path's types and defaults.  One
// deliberate difference: CHECK_CUDA (include/types.hpp:37-44) throws
// std::runtime_error carrying the CUDA error string, the file and the line,
// instead of printing and calling exit(1), so a failing CUDA call in a caller
// unwinds like every other error of this library.  CHECK_MPI is not provided:
// this single-GPU library has no MPI layer.
#ifndef HBDIA_B200_TYPES_HPP
#define HBDIA_B200_TYPES_HPP

#include <cuda_runtime_api.h>

#include <stdexcept>
#include <string>

// include/types.hpp:5
using DataType = double;

// COO remainder execution choice (include/types.hpp:7-10).  Accepted for
// source compatibility; the remainder always runs fused on the GPU.
enum class ExecutionMode {
    CPU_COO,
    GPU_COO
};

// include/types.hpp:14-21
#ifndef DEFAULT_BLOCK_WIDTH
#define DEFAULT_BLOCK_WIDTH 32
#endif
#ifndef DEFAULT_THRESHOLD
#define DEFAULT_THRESHOLD 1
#endif
#ifndef MAX_COO_ENTRIES
#define MAX_COO_ENTRIES 1000000000
#endif
#ifndef THREADS_PER_BLOCK_SPMV
#define THREADS_PER_BLOCK_SPMV 256
#endif
#ifndef THREADS_PER_BLOCK_VECTOR_ADD
#define THREADS_PER_BLOCK_VECTOR_ADD 256
#endif
#ifndef RAND_SEED
#define RAND_SEED 42
#endif
#ifndef NUM_BENCH_ITER
#define NUM_BENCH_ITER 100
#endif

#define CHECK_CUDA(call)                                                                                     \
    do {                                                                                                     \
        const cudaError_t hbdia_check_err_ = (call);                                                         \
        if (hbdia_check_err_ != cudaSuccess)                                                                 \
            throw std::runtime_error(std::string("CUDA error at ") + __FILE__ + ":" + std::to_string(__LINE__) + \
                                     " - " + cudaGetErrorString(hbdia_check_err_));                          \
    } while (0)

#endif
