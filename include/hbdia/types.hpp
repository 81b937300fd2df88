// Drop-in replacement for the reference's include/types.hpp (the parts the
// SpMV path uses).  CHECK_CUDA / CHECK_MPI are not provided: this library
// reports CUDA failures as exceptions (std::runtime_error) instead of
// exit(1), and has no MPI layer.
#ifndef HBDIA_B200_TYPES_HPP
#define HBDIA_B200_TYPES_HPP

// COO remainder execution choice (include/types.hpp:7-10).  Accepted for
// source compatibility; the remainder always runs fused on the GPU.
enum class ExecutionMode {
    CPU_COO,
    GPU_COO
};

// include/types.hpp:14-16
#ifndef DEFAULT_BLOCK_WIDTH
#define DEFAULT_BLOCK_WIDTH 32
#endif
#ifndef DEFAULT_THRESHOLD
#define DEFAULT_THRESHOLD 1
#endif
#ifndef MAX_COO_ENTRIES
#define MAX_COO_ENTRIES 1000000000
#endif

#endif
