// Drop-in hbdiaSpMV (reference: include/Operations/HBDIASpMV.hpp:8-10,
// src/Operations/HBDIASpMV.cpp:186-251).
//
// y = A x as ONE fused sm_100a launch (blocked-DIA part and COO remainder) on
// the matrix's stream; asynchronous like the reference (call
// matrix.synchronize() or cudaDeviceSynchronize()).  Returns true.  Throws
// std::runtime_error("Invalid COO execution flags") when the matrix has a COO
// remainder and both flags are false, as the reference does
// (src/Operations/HBDIASpMV.cpp:229-232); either flag selects the same GPU
// path.  Every row of y is written (the reference leaves rows of blocks
// without stored diagonals untouched, which differs only when y was not zero
// on entry).
#ifndef HBDIA_B200_HBDIASPMV_HPP
#define HBDIA_B200_HBDIASPMV_HPP

#include <cuda_runtime.h>

#include "../Format/HBDIA.hpp"
#include "../Format/HBDIAVector.hpp"

template <typename T>
bool hbdiaSpMV(HBDIA<T> &matrix, const HBDIAVector<T> &inputVector, HBDIAVector<T> &outputVector,
               bool execCooCPU, bool execCooGPU);

#endif
