/*
 * Drop-in declarations: the entry point of the reference header cudaICEEMDAN.cuh
 * (EEGLab-Pannon/CEEMDAN-GPU, cudaICEEMDAN.cuh:26), same name, arguments, C++ linkage
 * (mangled _Z9iceemdanDmmmmPiPdS0_d), device-pointer contract and [num_IMFs x N] output
 * layout.  A caller of the reference relinks against libceemdan_b200.so unchanged.
 *
 * Returns the elapsed seconds of the CEEMDAN stages (the reference's timer scope,
 * cudaICEEMDAN.cu:1723,2017-2018), or a negative value when the engine rejected the call
 * (-(double)ceemdan_status; the reference has no error reporting).
 * Noise: cuRAND XORWOW, seed 1234, as cudaICEEMDAN.cu:1460-1462.
 */
#pragma once
#include <stddef.h>

double iceemdanD(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                 int* d_x, double* d_y, double* d_IMFs, double noiseStrength);
