// Generated by gen_smem_layout.py: shared-memory sequence layout (padding
// shift SH, sequence stride SEQ) of the pass kernels, chosen per length and
// precision by replaying the kernels' shared-memory accesses through a bank
// model.  Element i of sequence s sits at s*SEQ + i + (SH ? i >> SH : 0).
#pragma once

namespace pb {

struct SmemLayout {
  int sh;
  int seq;
};

// pow2: {f32}, {f64} per length
__host__ __device__ constexpr SmemLayout pow2_layout(int N, int real_bytes) {
  switch (N) {
    case 32: return real_bytes == 4 ? SmemLayout{0, 35} : SmemLayout{2, 44};
    case 64: return real_bytes == 4 ? SmemLayout{2, 79} : SmemLayout{3, 71};
    case 128: return real_bytes == 4 ? SmemLayout{4, 135} : SmemLayout{3, 143};
    case 256: return real_bytes == 4 ? SmemLayout{4, 271} : SmemLayout{3, 287};
    case 512: return real_bytes == 4 ? SmemLayout{4, 546} : SmemLayout{3, 578};
    case 1024: return real_bytes == 4 ? SmemLayout{4, 1096} : SmemLayout{3, 1156};
    case 2048: return real_bytes == 4 ? SmemLayout{4, 2175} : SmemLayout{3, 2303};
    default: return SmemLayout{3, N + N / 8 + 1};
  }
}

// mr: {f32}, {f64} per length
__host__ __device__ constexpr SmemLayout mr_layout(int N, int real_bytes) {
  switch (N) {
    case 32: return real_bytes == 4 ? SmemLayout{0, 33} : SmemLayout{3, 39};
    case 35: return real_bytes == 4 ? SmemLayout{0, 35} : SmemLayout{0, 35};
    case 36: return real_bytes == 4 ? SmemLayout{2, 45} : SmemLayout{0, 37};
    case 40: return real_bytes == 4 ? SmemLayout{0, 53} : SmemLayout{0, 45};
    case 42: return real_bytes == 4 ? SmemLayout{0, 45} : SmemLayout{0, 43};
    case 45: return real_bytes == 4 ? SmemLayout{0, 45} : SmemLayout{0, 45};
    case 48: return real_bytes == 4 ? SmemLayout{0, 55} : SmemLayout{0, 49};
    case 49: return real_bytes == 4 ? SmemLayout{0, 49} : SmemLayout{0, 49};
    case 50: return real_bytes == 4 ? SmemLayout{0, 57} : SmemLayout{0, 55};
    case 54: return real_bytes == 4 ? SmemLayout{0, 69} : SmemLayout{0, 59};
    case 56: return real_bytes == 4 ? SmemLayout{0, 71} : SmemLayout{0, 63};
    case 60: return real_bytes == 4 ? SmemLayout{0, 63} : SmemLayout{2, 75};
    case 63: return real_bytes == 4 ? SmemLayout{0, 63} : SmemLayout{0, 63};
    case 64: return real_bytes == 4 ? SmemLayout{2, 79} : SmemLayout{3, 71};
    case 70: return real_bytes == 4 ? SmemLayout{0, 75} : SmemLayout{0, 75};
    case 72: return real_bytes == 4 ? SmemLayout{0, 73} : SmemLayout{0, 75};
    case 75: return real_bytes == 4 ? SmemLayout{0, 75} : SmemLayout{0, 75};
    case 80: return real_bytes == 4 ? SmemLayout{0, 87} : SmemLayout{0, 81};
    case 81: return real_bytes == 4 ? SmemLayout{0, 81} : SmemLayout{0, 81};
    case 84: return real_bytes == 4 ? SmemLayout{2, 105} : SmemLayout{0, 85};
    case 90: return real_bytes == 4 ? SmemLayout{0, 105} : SmemLayout{5, 99};
    case 96: return real_bytes == 4 ? SmemLayout{0, 97} : SmemLayout{0, 97};
    case 98: return real_bytes == 4 ? SmemLayout{0, 103} : SmemLayout{0, 103};
    case 100: return real_bytes == 4 ? SmemLayout{0, 109} : SmemLayout{2, 125};
    case 105: return real_bytes == 4 ? SmemLayout{0, 105} : SmemLayout{0, 105};
    case 108: return real_bytes == 4 ? SmemLayout{0, 121} : SmemLayout{0, 109};
    case 112: return real_bytes == 4 ? SmemLayout{4, 119} : SmemLayout{3, 127};
    case 120: return real_bytes == 4 ? SmemLayout{0, 121} : SmemLayout{3, 135};
    case 125: return real_bytes == 4 ? SmemLayout{0, 125} : SmemLayout{0, 125};
    case 126: return real_bytes == 4 ? SmemLayout{0, 137} : SmemLayout{0, 131};
    case 128: return real_bytes == 4 ? SmemLayout{4, 141} : SmemLayout{3, 143};
    case 135: return real_bytes == 4 ? SmemLayout{0, 135} : SmemLayout{0, 135};
    case 140: return real_bytes == 4 ? SmemLayout{0, 151} : SmemLayout{0, 147};
    case 144: return real_bytes == 4 ? SmemLayout{5, 149} : SmemLayout{0, 145};
    case 147: return real_bytes == 4 ? SmemLayout{0, 147} : SmemLayout{0, 147};
    case 150: return real_bytes == 4 ? SmemLayout{0, 153} : SmemLayout{0, 155};
    case 160: return real_bytes == 4 ? SmemLayout{0, 161} : SmemLayout{0, 161};
    case 162: return real_bytes == 4 ? SmemLayout{0, 175} : SmemLayout{5, 167};
    case 168: return real_bytes == 4 ? SmemLayout{5, 183} : SmemLayout{0, 171};
    case 175: return real_bytes == 4 ? SmemLayout{0, 175} : SmemLayout{0, 175};
    case 180: return real_bytes == 4 ? SmemLayout{2, 225} : SmemLayout{0, 181};
    case 189: return real_bytes == 4 ? SmemLayout{0, 189} : SmemLayout{0, 189};
    case 192: return real_bytes == 4 ? SmemLayout{2, 239} : SmemLayout{0, 193};
    case 196: return real_bytes == 4 ? SmemLayout{5, 202} : SmemLayout{2, 250};
    case 200: return real_bytes == 4 ? SmemLayout{3, 226} : SmemLayout{0, 202};
    case 210: return real_bytes == 4 ? SmemLayout{0, 210} : SmemLayout{0, 210};
    case 216: return real_bytes == 4 ? SmemLayout{5, 222} : SmemLayout{5, 222};
    case 224: return real_bytes == 4 ? SmemLayout{0, 238} : SmemLayout{3, 258};
    case 225: return real_bytes == 4 ? SmemLayout{0, 238} : SmemLayout{0, 230};
    case 240: return real_bytes == 4 ? SmemLayout{0, 242} : SmemLayout{0, 242};
    case 243: return real_bytes == 4 ? SmemLayout{0, 250} : SmemLayout{0, 246};
    case 245: return real_bytes == 4 ? SmemLayout{0, 250} : SmemLayout{0, 246};
    case 250: return real_bytes == 4 ? SmemLayout{0, 250} : SmemLayout{0, 250};
    case 252: return real_bytes == 4 ? SmemLayout{0, 266} : SmemLayout{5, 266};
    case 256: return real_bytes == 4 ? SmemLayout{4, 274} : SmemLayout{3, 290};
    case 270: return real_bytes == 4 ? SmemLayout{0, 270} : SmemLayout{0, 270};
    case 280: return real_bytes == 4 ? SmemLayout{0, 282} : SmemLayout{0, 282};
    case 288: return real_bytes == 4 ? SmemLayout{0, 290} : SmemLayout{0, 290};
    case 294: return real_bytes == 4 ? SmemLayout{0, 294} : SmemLayout{0, 294};
    case 300: return real_bytes == 4 ? SmemLayout{5, 318} : SmemLayout{0, 306};
    case 315: return real_bytes == 4 ? SmemLayout{0, 318} : SmemLayout{0, 318};
    case 320: return real_bytes == 4 ? SmemLayout{0, 322} : SmemLayout{0, 322};
    case 324: return real_bytes == 4 ? SmemLayout{0, 326} : SmemLayout{5, 334};
    case 336: return real_bytes == 4 ? SmemLayout{0, 338} : SmemLayout{0, 338};
    case 343: return real_bytes == 4 ? SmemLayout{0, 346} : SmemLayout{0, 346};
    case 350: return real_bytes == 4 ? SmemLayout{0, 350} : SmemLayout{0, 350};
    case 360: return real_bytes == 4 ? SmemLayout{0, 362} : SmemLayout{5, 378};
    case 375: return real_bytes == 4 ? SmemLayout{0, 378} : SmemLayout{0, 378};
    case 378: return real_bytes == 4 ? SmemLayout{0, 378} : SmemLayout{0, 378};
    case 384: return real_bytes == 4 ? SmemLayout{0, 386} : SmemLayout{0, 386};
    case 392: return real_bytes == 4 ? SmemLayout{0, 396} : SmemLayout{0, 396};
    case 400: return real_bytes == 4 ? SmemLayout{4, 428} : SmemLayout{3, 452};
    case 405: return real_bytes == 4 ? SmemLayout{0, 412} : SmemLayout{0, 412};
    case 420: return real_bytes == 4 ? SmemLayout{0, 420} : SmemLayout{2, 524};
    case 432: return real_bytes == 4 ? SmemLayout{4, 460} : SmemLayout{3, 492};
    case 441: return real_bytes == 4 ? SmemLayout{0, 444} : SmemLayout{0, 444};
    case 448: return real_bytes == 4 ? SmemLayout{0, 452} : SmemLayout{0, 452};
    case 450: return real_bytes == 4 ? SmemLayout{0, 460} : SmemLayout{0, 452};
    case 480: return real_bytes == 4 ? SmemLayout{4, 516} : SmemLayout{3, 540};
    case 486: return real_bytes == 4 ? SmemLayout{0, 492} : SmemLayout{0, 492};
    case 490: return real_bytes == 4 ? SmemLayout{0, 492} : SmemLayout{0, 492};
    case 500: return real_bytes == 4 ? SmemLayout{0, 500} : SmemLayout{2, 628};
    case 504: return real_bytes == 4 ? SmemLayout{3, 572} : SmemLayout{3, 572};
    case 512: return real_bytes == 4 ? SmemLayout{4, 548} : SmemLayout{3, 580};
    case 525: return real_bytes == 4 ? SmemLayout{0, 532} : SmemLayout{0, 532};
    case 540: return real_bytes == 4 ? SmemLayout{0, 540} : SmemLayout{0, 540};
    case 560: return real_bytes == 4 ? SmemLayout{0, 564} : SmemLayout{0, 564};
    case 567: return real_bytes == 4 ? SmemLayout{0, 572} : SmemLayout{0, 572};
    case 576: return real_bytes == 4 ? SmemLayout{0, 580} : SmemLayout{4, 612};
    case 588: return real_bytes == 4 ? SmemLayout{2, 740} : SmemLayout{0, 588};
    case 600: return real_bytes == 4 ? SmemLayout{0, 612} : SmemLayout{0, 604};
    case 625: return real_bytes == 4 ? SmemLayout{0, 628} : SmemLayout{0, 628};
    case 630: return real_bytes == 4 ? SmemLayout{0, 636} : SmemLayout{0, 636};
    case 640: return real_bytes == 4 ? SmemLayout{0, 644} : SmemLayout{0, 644};
    case 648: return real_bytes == 4 ? SmemLayout{3, 740} : SmemLayout{5, 668};
    case 672: return real_bytes == 4 ? SmemLayout{2, 844} : SmemLayout{0, 676};
    case 675: return real_bytes == 4 ? SmemLayout{0, 684} : SmemLayout{0, 676};
    case 686: return real_bytes == 4 ? SmemLayout{0, 692} : SmemLayout{0, 692};
    case 700: return real_bytes == 4 ? SmemLayout{0, 700} : SmemLayout{0, 700};
    case 720: return real_bytes == 4 ? SmemLayout{4, 764} : SmemLayout{0, 724};
    case 729: return real_bytes == 4 ? SmemLayout{0, 732} : SmemLayout{0, 732};
    case 735: return real_bytes == 4 ? SmemLayout{0, 740} : SmemLayout{0, 740};
    case 750: return real_bytes == 4 ? SmemLayout{0, 756} : SmemLayout{0, 756};
    case 756: return real_bytes == 4 ? SmemLayout{2, 948} : SmemLayout{0, 756};
    case 768: return real_bytes == 4 ? SmemLayout{2, 964} : SmemLayout{0, 772};
    case 770: return real_bytes == 4 ? SmemLayout{0, 780} : SmemLayout{0, 772};
    case 784: return real_bytes == 4 ? SmemLayout{0, 788} : SmemLayout{0, 788};
    case 800: return real_bytes == 4 ? SmemLayout{4, 852} : SmemLayout{3, 900};
    case 810: return real_bytes == 4 ? SmemLayout{0, 812} : SmemLayout{0, 812};
    case 840: return real_bytes == 4 ? SmemLayout{0, 852} : SmemLayout{0, 844};
    case 864: return real_bytes == 4 ? SmemLayout{4, 932} : SmemLayout{3, 972};
    case 875: return real_bytes == 4 ? SmemLayout{0, 876} : SmemLayout{0, 876};
    case 882: return real_bytes == 4 ? SmemLayout{0, 884} : SmemLayout{0, 884};
    case 896: return real_bytes == 4 ? SmemLayout{0, 900} : SmemLayout{0, 900};
    case 900: return real_bytes == 4 ? SmemLayout{0, 900} : SmemLayout{0, 900};
    case 945: return real_bytes == 4 ? SmemLayout{0, 948} : SmemLayout{0, 948};
    case 960: return real_bytes == 4 ? SmemLayout{4, 1020} : SmemLayout{3, 1084};
    case 972: return real_bytes == 4 ? SmemLayout{0, 972} : SmemLayout{0, 972};
    case 980: return real_bytes == 4 ? SmemLayout{0, 980} : SmemLayout{2, 1228};
    case 1000: return real_bytes == 4 ? SmemLayout{0, 1012} : SmemLayout{3, 1124};
    case 1008: return real_bytes == 4 ? SmemLayout{0, 1012} : SmemLayout{3, 1140};
    default: return SmemLayout{3, N + N / 8 + 1};
  }
}

}  // namespace pb
