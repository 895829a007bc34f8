/*
 * Drop-in declarations: the entry points of the reference header cudaICEEMDAN.cuh
 * (EEGLab-Pannon/CEEMDAN-GPU, cudaICEEMDAN.cuh:25-26), same names, arguments, C++ linkage
 * (mangled _Z9iceemdanSmmmmPiPfS0_f and _Z9iceemdanDmmmmPiPdS0_d), device-pointer contract and
 * [num_IMFs x N] output layout.  A caller of the reference relinks against libceemdan_b200.so
 * unchanged.
 *
 * Both return the elapsed seconds of the CEEMDAN stages (the reference's timer scope,
 * cudaICEEMDAN.cu:1723,2017-2018), or a negative value when the engine rejected the call
 * (-(double)ceemdan_status; the reference has no error reporting).
 * Noise: cuRAND XORWOW, seed 1234: float normals for iceemdanS (cudaICEEMDAN.cu:741), double
 * normals for iceemdanD (:1460-1462).
 * iceemdanS computes in FP64 on the exactly widened float data and noise and rounds the IMFs to
 * float (the reference computes in FP32).
 */
#pragma once
#include <stddef.h>

double iceemdanS(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                 int* d_x, float* d_y, float* d_IMFs, float noiseStrength);

double iceemdanD(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                 int* d_x, double* d_y, double* d_IMFs, double noiseStrength);
