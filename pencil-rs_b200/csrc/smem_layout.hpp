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
    case 32: return real_bytes == 4 ? SmemLayout{3, 38} : SmemLayout{0, 33};
    case 64: return real_bytes == 4 ? SmemLayout{2, 83} : SmemLayout{3, 71};
    case 128: return real_bytes == 4 ? SmemLayout{4, 135} : SmemLayout{4, 135};
    case 256: return real_bytes == 4 ? SmemLayout{4, 271} : SmemLayout{5, 263};
    case 512: return real_bytes == 4 ? SmemLayout{4, 546} : SmemLayout{5, 527};
    case 1024: return real_bytes == 4 ? SmemLayout{4, 1087} : SmemLayout{5, 1055};
    case 2048: return real_bytes == 4 ? SmemLayout{4, 2175} : SmemLayout{5, 2111};
    default: return SmemLayout{3, N + N / 8 + 1};
  }
}

// mr: {f32}, {f64} per length
__host__ __device__ constexpr SmemLayout mr_layout(int N, int real_bytes) {
  switch (N) {
    case 35: return real_bytes == 4 ? SmemLayout{5, 39} : SmemLayout{0, 37};
    case 36: return real_bytes == 4 ? SmemLayout{0, 41} : SmemLayout{5, 43};
    case 40: return real_bytes == 4 ? SmemLayout{0, 53} : SmemLayout{0, 45};
    case 42: return real_bytes == 4 ? SmemLayout{0, 53} : SmemLayout{0, 45};
    case 45: return real_bytes == 4 ? SmemLayout{0, 45} : SmemLayout{0, 45};
    case 48: return real_bytes == 4 ? SmemLayout{0, 51} : SmemLayout{0, 51};
    case 49: return real_bytes == 4 ? SmemLayout{5, 51} : SmemLayout{0, 55};
    case 50: return real_bytes == 4 ? SmemLayout{2, 63} : SmemLayout{5, 58};
    case 54: return real_bytes == 4 ? SmemLayout{0, 55} : SmemLayout{5, 58};
    case 56: return real_bytes == 4 ? SmemLayout{0, 71} : SmemLayout{0, 63};
    case 60: return real_bytes == 4 ? SmemLayout{2, 75} : SmemLayout{2, 75};
    case 63: return real_bytes == 4 ? SmemLayout{0, 73} : SmemLayout{5, 65};
    case 70: return real_bytes == 4 ? SmemLayout{0, 85} : SmemLayout{0, 74};
    case 72: return real_bytes == 4 ? SmemLayout{0, 85} : SmemLayout{3, 81};
    case 75: return real_bytes == 4 ? SmemLayout{0, 75} : SmemLayout{0, 75};
    case 80: return real_bytes == 4 ? SmemLayout{0, 85} : SmemLayout{0, 85};
    case 81: return real_bytes == 4 ? SmemLayout{0, 91} : SmemLayout{0, 83};
    case 84: return real_bytes == 4 ? SmemLayout{2, 105} : SmemLayout{0, 85};
    case 90: return real_bytes == 4 ? SmemLayout{0, 105} : SmemLayout{0, 90};
    case 96: return real_bytes == 4 ? SmemLayout{4, 102} : SmemLayout{5, 99};
    case 98: return real_bytes == 4 ? SmemLayout{0, 110} : SmemLayout{5, 102};
    case 100: return real_bytes == 4 ? SmemLayout{2, 125} : SmemLayout{2, 125};
    case 105: return real_bytes == 4 ? SmemLayout{0, 105} : SmemLayout{0, 107};
    case 108: return real_bytes == 4 ? SmemLayout{5, 111} : SmemLayout{2, 141};
    case 112: return real_bytes == 4 ? SmemLayout{0, 126} : SmemLayout{4, 119};
    case 120: return real_bytes == 4 ? SmemLayout{3, 135} : SmemLayout{0, 127};
    case 125: return real_bytes == 4 ? SmemLayout{0, 137} : SmemLayout{0, 125};
    case 126: return real_bytes == 4 ? SmemLayout{0, 138} : SmemLayout{5, 130};
    case 135: return real_bytes == 4 ? SmemLayout{0, 135} : SmemLayout{0, 141};
    case 140: return real_bytes == 4 ? SmemLayout{0, 147} : SmemLayout{2, 177};
    case 144: return real_bytes == 4 ? SmemLayout{0, 147} : SmemLayout{3, 162};
    case 147: return real_bytes == 4 ? SmemLayout{0, 149} : SmemLayout{0, 149};
    case 150: return real_bytes == 4 ? SmemLayout{0, 158} : SmemLayout{0, 150};
    case 160: return real_bytes == 4 ? SmemLayout{0, 165} : SmemLayout{2, 201};
    case 162: return real_bytes == 4 ? SmemLayout{0, 166} : SmemLayout{0, 166};
    case 168: return real_bytes == 4 ? SmemLayout{0, 181} : SmemLayout{3, 189};
    case 175: return real_bytes == 4 ? SmemLayout{0, 179} : SmemLayout{0, 179};
    case 180: return real_bytes == 4 ? SmemLayout{2, 225} : SmemLayout{0, 180};
    case 189: return real_bytes == 4 ? SmemLayout{0, 189} : SmemLayout{0, 191};
    case 192: return real_bytes == 4 ? SmemLayout{0, 195} : SmemLayout{3, 215};
    case 196: return real_bytes == 4 ? SmemLayout{0, 204} : SmemLayout{2, 251};
    case 200: return real_bytes == 4 ? SmemLayout{4, 218} : SmemLayout{3, 225};
    case 210: return real_bytes == 4 ? SmemLayout{0, 210} : SmemLayout{0, 210};
    case 216: return real_bytes == 4 ? SmemLayout{4, 236} : SmemLayout{3, 243};
    case 224: return real_bytes == 4 ? SmemLayout{0, 236} : SmemLayout{4, 238};
    case 225: return real_bytes == 4 ? SmemLayout{0, 237} : SmemLayout{0, 225};
    case 240: return real_bytes == 4 ? SmemLayout{4, 263} : SmemLayout{3, 270};
    case 243: return real_bytes == 4 ? SmemLayout{0, 257} : SmemLayout{0, 249};
    case 245: return real_bytes == 4 ? SmemLayout{0, 259} : SmemLayout{0, 251};
    case 250: return real_bytes == 4 ? SmemLayout{0, 258} : SmemLayout{0, 250};
    case 252: return real_bytes == 4 ? SmemLayout{4, 270} : SmemLayout{2, 315};
    case 270: return real_bytes == 4 ? SmemLayout{0, 282} : SmemLayout{0, 274};
    case 280: return real_bytes == 4 ? SmemLayout{0, 294} : SmemLayout{3, 315};
    case 288: return real_bytes == 4 ? SmemLayout{0, 292} : SmemLayout{3, 324};
    case 294: return real_bytes == 4 ? SmemLayout{0, 298} : SmemLayout{0, 298};
    case 300: return real_bytes == 4 ? SmemLayout{0, 300} : SmemLayout{0, 300};
    case 315: return real_bytes == 4 ? SmemLayout{0, 330} : SmemLayout{0, 321};
    case 320: return real_bytes == 4 ? SmemLayout{0, 334} : SmemLayout{3, 365};
    case 324: return real_bytes == 4 ? SmemLayout{5, 334} : SmemLayout{0, 324};
    case 336: return real_bytes == 4 ? SmemLayout{0, 340} : SmemLayout{3, 378};
    case 343: return real_bytes == 4 ? SmemLayout{5, 354} : SmemLayout{0, 345};
    case 350: return real_bytes == 4 ? SmemLayout{0, 358} : SmemLayout{0, 350};
    case 360: return real_bytes == 4 ? SmemLayout{0, 365} : SmemLayout{3, 405};
    case 375: return real_bytes == 4 ? SmemLayout{0, 390} : SmemLayout{0, 379};
    case 378: return real_bytes == 4 ? SmemLayout{0, 390} : SmemLayout{0, 382};
    case 384: return real_bytes == 4 ? SmemLayout{5, 396} : SmemLayout{3, 431};
    case 392: return real_bytes == 4 ? SmemLayout{0, 392} : SmemLayout{0, 393};
    case 400: return real_bytes == 4 ? SmemLayout{4, 425} : SmemLayout{3, 450};
    case 405: return real_bytes == 4 ? SmemLayout{0, 420} : SmemLayout{0, 407};
    case 420: return real_bytes == 4 ? SmemLayout{0, 420} : SmemLayout{2, 525};
    case 432: return real_bytes == 4 ? SmemLayout{4, 459} : SmemLayout{4, 459};
    case 441: return real_bytes == 4 ? SmemLayout{0, 451} : SmemLayout{0, 447};
    case 448: return real_bytes == 4 ? SmemLayout{0, 456} : SmemLayout{0, 449};
    case 450: return real_bytes == 4 ? SmemLayout{0, 458} : SmemLayout{2, 563};
    case 480: return real_bytes == 4 ? SmemLayout{4, 516} : SmemLayout{3, 540};
    case 486: return real_bytes == 4 ? SmemLayout{0, 498} : SmemLayout{2, 611};
    case 490: return real_bytes == 4 ? SmemLayout{0, 502} : SmemLayout{2, 612};
    case 500: return real_bytes == 4 ? SmemLayout{0, 500} : SmemLayout{2, 629};
    case 504: return real_bytes == 4 ? SmemLayout{4, 540} : SmemLayout{3, 567};
    default: return SmemLayout{3, N + N / 8 + 1};
  }
}

}  // namespace pb
