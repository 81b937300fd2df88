// Drop-in HBDIAVector<T> (reference: include/Format/HBDIAVector.hpp:23-109)
// on one GPU: a device buffer holding the local vector.  With no halo parts
// the data and local pointers coincide.
//
// The reference's unified-memory constructor (HBDIAVector.hpp:32) is kept
// for source compatibility: its four flags are accepted and the vector lives
// in device memory all the same, which is where the fused SpMV reads and
// writes fastest (the reference's flags select malloc / managed / NUMA host
// allocations for a Grace-Hopper node's shared memory).  getDeviceCOOResultsPtr
// (HBDIAVector.hpp:53) returns a zeroed buffer of the vector's length that
// callers may clear as they do for the reference; the fused SpMV writes y once
// and never uses it.
#ifndef HBDIA_B200_HBDIAVECTOR_HPP
#define HBDIA_B200_HBDIAVECTOR_HPP

#include <cstddef>
#include <vector>

#include "HBDIA.hpp"

template <typename T>
class HBDIAVector {
public:
    HBDIAVector();
    explicit HBDIAVector(const std::vector<T> &localData);
    HBDIAVector(const std::vector<T> &localData, bool unifiedMemory, bool unifiedMemoryMalloc,
                bool unifiedMemoryManagedMalloc, bool unifiedNumaAllocOnNode);
    ~HBDIAVector();
    HBDIAVector(const HBDIAVector &) = delete;
    HBDIAVector &operator=(const HBDIAVector &) = delete;
    HBDIAVector(HBDIAVector &&other) noexcept;
    HBDIAVector &operator=(HBDIAVector &&other) noexcept;

    const std::vector<T> &getLocalVector() const { return localVector_; }
    size_t getLocalSize() const { return localVector_.size(); }
    size_t getTotalSize() const { return localVector_.size(); }
    T *getDeviceDataPtr() const;
    T *getDeviceLocalPtr() const { return getDeviceDataPtr(); }
    T *getDeviceCOOResultsPtr() const;

    // blocking copies between the device buffer and host memory
    void copyToHost(std::vector<T> &out) const;
    void copyFromHost(const std::vector<T> &in);

    hbdia_vector *handle() const { return h_; }

private:
    std::vector<T> localVector_;
    hbdia_vector *h_ = nullptr;
};

#endif
