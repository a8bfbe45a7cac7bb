// Line lengths served by the mixed-radix pass kernel (mr_kernel.cuh): the
// 115 numbers 2^a 3^b 5^c 7^d in [35, 1008] that are not powers of two.  The
// kernels are split over MR_GROUPS translation units (mr_kernels.cu compiled
// once per group) so that they build in parallel.
#pragma once

#include <cuda_runtime.h>

#include "pb_internal.hpp"

namespace pb {

constexpr int kMrLengths[] = {35,  36,  40,  42,  45,  48,  49,  50,  54,  56,  60,  63,  70,  72,  75,  80,
                              81,  84,  90,  96,  98,  100, 105, 108, 112, 120, 125, 126, 135, 140, 144, 147,
                              150, 160, 162, 168, 175, 180, 189, 192, 196, 200, 210, 216, 224, 225, 240, 243,
                              245, 250, 252, 270, 280, 288, 294, 300, 315, 320, 324, 336, 343, 350, 360, 375,
                              378, 384, 392, 400, 405, 420, 432, 441, 448, 450, 480, 486, 490, 500, 504,
                              525, 540, 560, 567, 576, 588, 600, 625, 630, 640, 648, 672, 675, 686, 700, 720,
                              729, 735, 750, 756, 768, 784, 800, 810, 840, 864, 875, 882, 896, 900, 945, 960,
                              972, 980, 1000, 1008};
constexpr int kMrCount = sizeof(kMrLengths) / sizeof(kMrLengths[0]);

// Resident CTAs per SM the kernels are compiled for (the register budget
// 65536 / (256 threads x CTAs): 128 registers at 2, 80 at 3).  f32 lengths up
// to 512 take 3: more warps hide the shared-memory and barrier latency that
// bounds these kernels (a per-length sweep of 2^25-element C2C and R2C passes:
// 0.82-0.95 of the 2-CTA time on most lengths; the real-to-real kinds
// 0.70-0.90 on every length).  The exceptions below keep 2 with the default
// schedule: their radix-16 and radix-15 stages spill at 80 registers and lost
// (1.02-1.37x) in that sweep.  f64 and lengths above 512 keep 2.
constexpr int kMrTwoCtaLengths[] = {45, 75, 81, 90, 135, 160, 168, 180, 192, 196, 210, 216, 224, 225, 240, 360};

__host__ __device__ constexpr bool mr_two_cta_length(int N) {
  for (int n : kMrTwoCtaLengths)
    if (n == N) return true;
  return false;
}

// Lengths above 512 whose default-schedule f32 kernel fits 80 registers, so
// three CTAs per SM, without spilling (the strided and split-store variants
// spill at most 16 bytes); the other long lengths spill 40-650 bytes there.
constexpr int kMrThreeCtaLongLengths[] = {525, 540, 567, 576};

__host__ __device__ constexpr bool mr_three_cta_long_length(int N) {
  for (int n : kMrThreeCtaLongLengths)
    if (n == N) return true;
  return false;
}

// CTAs per SM of the mixed-radix kernel for precision `real_bytes`, length N
// and schedule S (1: radices up to 8, fewer registers per butterfly).
__host__ __device__ constexpr int mr_min_ctas(int real_bytes, int N, int S) {
  return real_bytes != 4 ? 2
         : N > 512       ? ((S == 0 && mr_three_cta_long_length(N)) ? 3 : 2)
                         : (S == 1 ? 3 : (mr_two_cta_length(N) ? 2 : 3));
}

// The same for the real-to-real kinds (default schedule only).  The 770-point
// kernel (the DST-I of a 384-point axis) takes 3 as well: with its row tables
// sized for the DST-I's outputs (mr_r2r_table_len) three CTAs fit in shared
// memory.
__host__ __device__ constexpr int mr_r2r_min_ctas(int real_bytes, int N) {
  return (real_bytes == 4 && (N <= 512 || N == 770)) ? 3 : 2;
}

// Outputs per line that the real-to-real kernel's row tables hold for FFT
// length N: 2N up to 512 (the type-IV kinds write n = 2N outputs from an
// N-point FFT), N above (770 serves the DST-I of 384, 384 outputs).  The host
// keeps passes with more outputs on the generic kernel.
__host__ __device__ constexpr int mr_r2r_table_len(int N) { return N <= 512 ? 2 * N : N; }
constexpr int MR_GROUPS = 8;

// Convolution lengths of Bluestein passes up to 1024 points: the smallest entry
// >= 2m - 1 is taken (powers of two and 7-smooth lengths between them, so
// that the convolution stays within about 1.8x of 2m); mr_bs.cuh is
// instantiated for each.  Longer convolutions (generic kernel only) are powers
// of two.
constexpr int kBluesteinLengths[] = {80,  96,  112, 128, 160, 192, 224, 256, 288,
                                     320, 384, 448, 512, 576, 640, 768, 896, 1024};
constexpr int kBluesteinCount = sizeof(kBluesteinLengths) / sizeof(kBluesteinLengths[0]);

// Lengths whose passes the persistent batch kernel (pass_kernel.cu) runs with
// the mixed-radix tile code, f32 only: the 7-smooth numbers in [32, 256],
// powers of two included.  Other passes of a batch take the generic tile code.
constexpr int kBatchMrLengths[] = {32,  35,  36,  40,  42,  45,  48,  49,  50,  54,  56,  60,  63,  64,
                                   70,  72,  75,  80,  81,  84,  90,  96,  98,  100, 105, 108, 112, 120,
                                   125, 126, 128, 135, 140, 144, 147, 150, 160, 162, 168, 175, 180, 189,
                                   192, 196, 200, 210, 216, 224, 225, 240, 243, 245, 250, 252, 256};
constexpr int kBatchMrCount = sizeof(kBatchMrLengths) / sizeof(kBatchMrLengths[0]);

// FFT lengths of the real-to-real kinds on the mixed-radix kernel
// (mr_r2r.cuh): the mixed-radix lengths, the powers of two 32..512, and 770
// (= 2(384 + 1), the DST-I extension of a 384-point axis; radix 11).
constexpr int kMrR2rLengths[] = {32,  35,  36,  40,  42,  45,  48,  49,  50,  54,  56,  60,  63,  64,  70,  72,  75,
                                 80,  81,  84,  90,  96,  98,  100, 105, 108, 112, 120, 125, 126, 128, 135, 140, 144,
                                 147, 150, 160, 162, 168, 175, 180, 189, 192, 196, 200, 210, 216, 224, 225, 240, 243,
                                 245, 250, 252, 256, 270, 280, 288, 294, 300, 315, 320, 324, 336, 343, 350, 360, 375,
                                 378, 384, 392, 400, 405, 420, 432, 441, 448, 450, 480, 486, 490, 500, 504, 512, 770};
constexpr int kMrR2rCount = sizeof(kMrR2rLengths) / sizeof(kMrR2rLengths[0]);

// Entry points of one (precision, length) instantiation.
struct MrEntry {
  cudaError_t (*launch)(const PassArgs&, cudaStream_t);
  int (*occupancy)(int sched);  // resident CTAs per SM of a schedule
  int nseq;                     // complex sequences per tile
  int nsched;                   // schedules available (1 or 2)
  int nrad[2];                  // stages of each schedule
  int rad[2][12];               // their radices, stage 0 first
};

// Filled by group g: entries i with i % MR_GROUPS == g of both tables.
void mr_fill_group0(MrEntry* f32, MrEntry* f64);
void mr_fill_group1(MrEntry* f32, MrEntry* f64);
void mr_fill_group2(MrEntry* f32, MrEntry* f64);
void mr_fill_group3(MrEntry* f32, MrEntry* f64);
void mr_fill_group4(MrEntry* f32, MrEntry* f64);
void mr_fill_group5(MrEntry* f32, MrEntry* f64);
void mr_fill_group6(MrEntry* f32, MrEntry* f64);
void mr_fill_group7(MrEntry* f32, MrEntry* f64);
// the real-to-real tables (kMrR2rLengths), filled by mr_r2r_kernels.cu
void mr_r2r_fill_group0(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group1(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group2(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group3(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group4(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group5(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group6(MrEntry* f32, MrEntry* f64);
void mr_r2r_fill_group7(MrEntry* f32, MrEntry* f64);

}  // namespace pb
