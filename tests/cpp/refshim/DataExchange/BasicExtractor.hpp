// Test fixture, not part of the library.  The reference's single-GPU
// programs include its MPI DataExchange headers (include/DataExchange/BasicExtractor.hpp)
// without using them on their single-GPU path; this library has no MPI
// layer, so the recipe that compiles those programs against include/hbdia/
// puts this empty header where the reference's stood.
#pragma once
