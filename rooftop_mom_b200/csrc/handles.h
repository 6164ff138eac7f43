// The opaque handles of the C ABI (include/rtm.h), shared by capi.cpp and server.cpp.
#pragma once

#include <memory>
#include <vector>

#include "grid.h"
#include "ops.h"

struct rtm_generators {
    rtm::DeviceGenerators g;
    int device = 0;
    cudaStream_t stream = nullptr;
    ~rtm_generators() {
        if (stream) cudaStreamSynchronize(stream);
        g.xx.reset();
        g.yy.reset();
        g.e.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

struct rtm_operator {
    std::unique_ptr<rtm::LinearOp> op;
    rtm::GridApplicator* grid = nullptr;  // the same object when the product is an FFT product
    int kind = 0;                    // rtm_product, or -1 for a dense matrix
    int device = 0;
    cudaStream_t stream = nullptr;
    ~rtm_operator() {
        if (stream) cudaStreamSynchronize(stream);
        op.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

struct rtm_preconditioner {
    std::unique_ptr<rtm::LinearOp> op;
    int device = 0;
    cudaStream_t stream = nullptr;
    ~rtm_preconditioner() {
        if (stream) cudaStreamSynchronize(stream);
        op.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace rtm {
// The rooftops of the middle port of a grid in direction 0 (x) or 1 (y), generateMiddlePort.m:14-28.
int middle_port(int count_x, int count_y, int direction, std::vector<int64_t>& port);
// RTM_OK when the direction and polarization of a plane wave are perpendicular unit vectors (to 1e-9), the
// form generatePlaneWave.m:18-42 takes them in (Excitation.planeWave normalises and checks them,
// Excitation.m:52-62); RTM_ERR_ARG otherwise.
int check_plane_wave(const double* direction, const double* polarization);
}  // namespace rtm
