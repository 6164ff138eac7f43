// Excitations and results on the device (excitation.cu).
#pragma once

#include "internal.h"

namespace rtm {

int plane_wave(int cx, int cy, double a, double b, int order, double k, const double* dirs, const double* pols,
               const double* intens, int nrhs, double2* out_device, cudaStream_t s);
int radar_cross_section(double k, const double2* e, const double2* J, int64_t n, double intensity, double* out,
                        cudaStream_t s);
int input_impedance(int cx, int cy, double a, double b, const double2* J, const int64_t* port_host, int count,
                    double voltage, double* out_re_im, cudaStream_t s);

}  // namespace rtm
