// The C ABI's matrix and vector handles (shared by the C ABI and the server).
#pragma once

#include <cstdint>
#include <mutex>

#include "hbdia_internal.hpp"

struct hbdia_vector {
    int32_t dtype = HBDIA_F64;
    int64_t n = 0;
    void *d = nullptr;
    void *cooResult = nullptr;  // getDeviceCOOResultsPtr's buffer (first request)
};

struct hbdia_matrix {
    int32_t dtype = HBDIA_F64;
    bool hasCOO = false;
    bool hasHBDIA = false;
    bool hostLayout = false;  // host layout materialised
    hbdia::Coo<double> c64;
    hbdia::Coo<float> c32;
    hbdia::HostLayout<double> L64;
    hbdia::HostLayout<float> L32;
    hbdia::DevicePlan plan;
    int32_t *blockSizesDev = nullptr;   // getBlockSizesDevice (first request; freed with the plan)
    hbdia::DeviceLayoutMeta devMeta;    // layout facts when the GPU converter built the plan
    bool hasDIA = false;                // DIA format (host data)
    std::vector<int32_t> diaOffsets;
    std::vector<double> dia64;
    std::vector<float> dia32;
    int32_t diaLength = 0;
    hbdia::DevicePlan innerPlan;        // reduced-storage copy for the CG inner iterations
    hbdia::CgWork *cg = nullptr;        // CG workspace
    int32_t blockWidth = 0, threshold = 0;
    int64_t maxCoo = 0;
    hbdia::PartialMeta part;            // partial matrix (one rank's rows) and its metadata
    // hbdia_spmv_host_many: device staging pairs and streams of its pipeline
    static constexpr int kHostDepth = 3;
    void *pipeX[kHostDepth] = {}, *pipeY[kHostDepth] = {}, *pipeStream[kHostDepth] = {};
    std::mutex hostMu;  // serialises hbdia_spmv_host's scratch buffers
};
