// castro_tuned.h -- launch shape of the fused batched step, chosen by
// mini-castro_b200/autotune.py from timings of the batched step
// (sedov128_pert) on the GPU it ran on.  Timing table (ms per step):
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.488
//   block64_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    4.077
//   block256_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    4.852
//   block128_minbeos0_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.597
//   block128_minbeos2_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.886
//   block128_minbeos3_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.594
//   block128_minbeos4_minbr32_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.564
//   block128_minbeos4_minbr33_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.566
//   block128_minbeos4_minbr34_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.488
//   block128_minbeos4_minbr30_minbriemann5_minbtrace0_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.495
//   block128_minbeos4_minbr30_minbriemann5_minbtrace2_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.623
//   block128_minbeos4_minbr30_minbriemann5_minbtrace4_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.540
//   block128_minbeos4_minbr30_minbriemann0_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.560
//   block128_minbeos4_minbr30_minbriemann3_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.574
//   block128_minbeos4_minbr30_minbriemann4_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.573
//   block128_minbeos4_minbr30_minbriemann6_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.551
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg3_tracesplit1    3.526
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg7_tracesplit1    3.493
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg9_tracesplit1    3.523
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit0    3.561
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace26_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.496
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace28_r2rows1_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.494
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage0_r3rows2_r3stage1_traceseg5_tracesplit1    3.645
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows2_r3stage0_traceseg5_tracesplit1    3.517
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows2_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.483
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows4_r2stage1_r3rows2_r3stage1_traceseg5_tracesplit1    3.515
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows1_r3stage1_traceseg5_tracesplit1    3.611
//   block128_minbeos4_minbr30_minbriemann5_minbtrace3_minbtrace20_r2rows1_r2stage1_r3rows4_r3stage1_traceseg5_tracesplit1    3.511
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
#define CASTRO_MINB_TRACE 3
#endif
#ifndef CASTRO_MINB_TRACE2
#define CASTRO_MINB_TRACE2 0
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
#ifndef CASTRO_TRACE_SPLIT
#define CASTRO_TRACE_SPLIT 1
#endif
#endif
