// castro_tuned.h -- launch shape of the fused batched step, chosen by
// mini-castro_b200/autotune.py from timings of the batched step
// (sedov128_pert) on the GPU it ran on.  Timing table (ms per step):
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.793
//   block64_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    4.468
//   block256_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    5.590
//   block128_minbeos0_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.851
//   block128_minbeos2_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    4.179
//   block128_minbeos3_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.853
//   block128_minbeos4_minbr32_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    4.072
//   block128_minbeos4_minbr33_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.889
//   block128_minbeos4_minbr34_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.940
//   block128_minbeos4_minbr30_minbriemann5_minbtrace0_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    4.033
//   block128_minbeos4_minbr30_minbriemann5_minbtrace2_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    4.033
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.794
//   block128_minbeos4_minbr30_minbriemann0_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.864
//   block128_minbeos4_minbr30_minbriemann3_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.880
//   block128_minbeos4_minbr30_minbriemann4_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.879
//   block128_minbeos4_minbr30_minbriemann6_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5    3.857
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg3    3.826
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg7    3.815
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage0_traceseg9    3.844
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage0_r3rows2_r3stage0_traceseg5    3.951
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5    3.767
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows2_r2stage1_r3rows2_r3stage1_traceseg5    3.760
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows4_r2stage1_r3rows2_r3stage1_traceseg5    3.792
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows1_r3stage1_traceseg5    3.889
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_r2rows1_r2stage1_r3rows4_r3stage1_traceseg5    3.785
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
#ifndef CASTRO_R2_ROWS
#define CASTRO_R2_ROWS 1
#endif
#ifndef CASTRO_R2_STAGE
#define CASTRO_R2_STAGE 1
#endif
#ifndef CASTRO_R3_ROWS
#define CASTRO_R3_ROWS 2
#endif
#ifndef CASTRO_R3_STAGE
#define CASTRO_R3_STAGE 1
#endif
#ifndef CASTRO_TRACE_SEG
#define CASTRO_TRACE_SEG 5
#endif
#endif
