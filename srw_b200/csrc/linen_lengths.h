// General FFT lengths with a specialised line-pass kernel (linen.cuh): 2^a m, a >= 4, for the odd parts
// m that range / resolution factors of 1.25, 1.5, 1.75 and their products give on 256 .. 1024-point
// inputs (3, 5, 7, 9, 15, 25, 35), from 320 to 7168 points.  Each is compiled as its own unit
// (linen.cu with SRWG_LINEN=N); other general lengths run the run-time-scheduled pass (lineg.cuh).
// The powers of two are compiled as well: the autotuner chooses, per axis and length, between them
// and the power-of-two pass (line2.cuh).
#pragma once

#define SRWG_LINEN_LENGTHS(X)                                                                            \
    X(320) X(384) X(400) X(448) X(480) X(560) X(576) X(640) X(768) X(800) X(896) X(960) X(1120) X(1152) \
    X(1280) X(1536) X(1600) X(1792) X(1920) X(2240) X(2304) X(2560) X(3072) X(3200) X(3584) X(3840)     \
    X(4480) X(4608) X(5120) X(6144) X(6400) X(7168)

#define SRWG_LINEN_POW2(X) X(256) X(512) X(1024) X(2048) X(4096) X(8192)
