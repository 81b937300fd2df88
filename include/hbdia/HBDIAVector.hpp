// Drop-in HBDIAVector<T> (reference: include/Format/HBDIAVector.hpp:23-109)
// on one GPU: a device buffer holding the local vector.  With no halo parts
// the data and local pointers coincide.  The reference's unified-memory
// variants and its separate COO-result buffer are not needed: the fused SpMV
// writes y once.
#ifndef HBDIA_B200_HBDIAVECTOR_HPP
#define HBDIA_B200_HBDIAVECTOR_HPP

#include <cstddef>
#include <vector>

#include "hbdia_b200.h"

template <typename T>
class HBDIAVector {
public:
    HBDIAVector();
    explicit HBDIAVector(const std::vector<T> &localData);
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

    // blocking copies between the device buffer and host memory
    void copyToHost(std::vector<T> &out) const;
    void copyFromHost(const std::vector<T> &in);

    hbdia_vector *handle() const { return h_; }

private:
    std::vector<T> localVector_;
    hbdia_vector *h_ = nullptr;
};

#endif
