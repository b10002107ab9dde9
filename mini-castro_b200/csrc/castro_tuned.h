// castro_tuned.h -- launch shape of the fused batched step, chosen by
// mini-castro_b200/autotune.py from timings of the batched step
// (sedov128_pert) on the GPU it ran on.  Timing table (ms per step):
//   block128_eos4_r30_riemann0_trace4_seg5      4.612
//   block64_eos4_r30_riemann0_trace4_seg5       5.226
//   block256_eos4_r30_riemann0_trace4_seg5      6.406
//   block128_eos0_r30_riemann0_trace4_seg5      4.670
//   block128_eos2_r30_riemann0_trace4_seg5      4.989
//   block128_eos3_r30_riemann0_trace4_seg5      4.667
//   block128_eos4_r32_riemann0_trace4_seg5      4.955
//   block128_eos4_r33_riemann0_trace4_seg5      4.654
//   block128_eos4_r34_riemann0_trace4_seg5      4.674
//   block128_eos4_r30_riemann0_trace0_seg5      4.910
//   block128_eos4_r30_riemann0_trace2_seg5      4.908
//   block128_eos4_r30_riemann0_trace3_seg5      4.623
//   block128_eos4_r30_riemann2_trace4_seg5      4.878
//   block128_eos4_r30_riemann3_trace4_seg5      4.879
//   block128_eos4_r30_riemann4_trace4_seg5      4.653
//   block128_eos4_r30_riemann0_trace4_seg3      4.660
//   block128_eos4_r30_riemann0_trace4_seg7      4.632
//   block128_eos4_r30_riemann0_trace4_seg9      4.675
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
#define CASTRO_MINB_TRACE 4
#endif
#ifndef CASTRO_TRACE_SEG
#define CASTRO_TRACE_SEG 5
#endif
#endif
