// castro_tuned.h -- launch shape of the fused batched step, chosen by
// mini-castro_b200/autotune.py from timings of the batched step
// (sedov128_pert) on the GPU it ran on.  Timing table (ms per step):
//   block128_eos4_r30_riemann5_trace4_stage1_stage0_seg5    4.288
//   block64_eos4_r30_riemann5_trace4_stage1_stage0_seg5    5.018
//   block256_eos4_r30_riemann5_trace4_stage1_stage0_seg5    6.347
//   block128_eos0_r30_riemann5_trace4_stage1_stage0_seg5    4.351
//   block128_eos2_r30_riemann5_trace4_stage1_stage0_seg5    4.668
//   block128_eos3_r30_riemann5_trace4_stage1_stage0_seg5    4.346
//   block128_eos4_r32_riemann5_trace4_stage1_stage0_seg5    4.599
//   block128_eos4_r33_riemann5_trace4_stage1_stage0_seg5    4.297
//   block128_eos4_r34_riemann5_trace4_stage1_stage0_seg5    4.322
//   block128_eos4_r30_riemann5_trace0_stage1_stage0_seg5    4.589
//   block128_eos4_r30_riemann5_trace2_stage1_stage0_seg5    4.586
//   block128_eos4_r30_riemann5_trace3_stage1_stage0_seg5    4.302
//   block128_eos4_r30_riemann0_trace4_stage1_stage0_seg5    4.369
//   block128_eos4_r30_riemann3_trace4_stage1_stage0_seg5    4.390
//   block128_eos4_r30_riemann4_trace4_stage1_stage0_seg5    4.390
//   block128_eos4_r30_riemann6_trace4_stage1_stage0_seg5    4.340
//   block128_eos4_r30_riemann5_trace4_stage1_stage0_seg3    4.337
//   block128_eos4_r30_riemann5_trace4_stage1_stage0_seg7    4.308
//   block128_eos4_r30_riemann5_trace4_stage1_stage0_seg9    4.353
//   block128_eos4_r30_riemann5_trace4_stage0_stage0_seg5    4.467
//   block128_eos4_r30_riemann5_trace4_stage1_stage1_seg5    4.336
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
#define CASTRO_MINB_RIEMANN 5
#endif
#ifndef CASTRO_MINB_TRACE
#define CASTRO_MINB_TRACE 4
#endif
#ifndef CASTRO_R2_STAGE
#define CASTRO_R2_STAGE 1
#endif
#ifndef CASTRO_R3_STAGE
#define CASTRO_R3_STAGE 0
#endif
#ifndef CASTRO_TRACE_SEG
#define CASTRO_TRACE_SEG 5
#endif
#endif
