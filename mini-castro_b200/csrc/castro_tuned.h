// castro_tuned.h -- launch shape of the fused batched step, chosen by
// mini-castro_b200/autotune.py from timings of the batched step
// (sedov128_pert) on the GPU it ran on.  Timing table (ms per step):
//   block128_eos4_r33_riemann0_trace0           4.750
//   block64_eos4_r33_riemann0_trace0            5.374
//   block256_eos4_r33_riemann0_trace0           5.479
//   block128_eos0_r33_riemann0_trace0           4.809
//   block128_eos2_r33_riemann0_trace0           5.129
//   block128_eos3_r33_riemann0_trace0           4.806
//   block128_eos4_r30_riemann0_trace0           4.699
//   block128_eos4_r32_riemann0_trace0           5.051
//   block128_eos4_r34_riemann0_trace0           4.769
//   block128_eos4_r30_riemann0_trace2           4.749
//   block128_eos4_r30_riemann0_trace3           4.749
//   block128_eos4_r30_riemann0_trace4           4.760
//   block128_eos4_r30_riemann2_trace0           4.981
//   block128_eos4_r30_riemann3_trace0           4.980
//   block128_eos4_r30_riemann4_trace0           4.747
#pragma once
#ifndef CASTRO_NO_TUNED_HEADER
#ifndef CASTRO_BLOCK
#define CASTRO_BLOCK 128
#endif
#ifndef CASTRO_MINB_EOS
#define CASTRO_MINB_EOS 4
#endif
#ifndef CASTRO_MINB_R3
#define CASTRO_MINB_R3 0
#endif
#ifndef CASTRO_MINB_RIEMANN
#define CASTRO_MINB_RIEMANN 0
#endif
#ifndef CASTRO_MINB_TRACE
#define CASTRO_MINB_TRACE 0
#endif
#endif
