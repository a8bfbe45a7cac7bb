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
    case 32: return real_bytes == 4 ? SmemLayout{0, 35} : SmemLayout{0, 33};
    case 35: return real_bytes == 4 ? SmemLayout{5, 39} : SmemLayout{0, 37};
    case 36: return real_bytes == 4 ? SmemLayout{2, 45} : SmemLayout{0, 43};
    case 40: return real_bytes == 4 ? SmemLayout{0, 53} : SmemLayout{0, 45};
    case 42: return real_bytes == 4 ? SmemLayout{0, 43} : SmemLayout{3, 47};
    case 45: return real_bytes == 4 ? SmemLayout{0, 45} : SmemLayout{0, 45};
    case 48: return real_bytes == 4 ? SmemLayout{0, 59} : SmemLayout{0, 55};
    case 49: return real_bytes == 4 ? SmemLayout{5, 51} : SmemLayout{0, 55};
    case 50: return real_bytes == 4 ? SmemLayout{5, 58} : SmemLayout{5, 58};
    case 54: return real_bytes == 4 ? SmemLayout{4, 57} : SmemLayout{5, 58};
    case 56: return real_bytes == 4 ? SmemLayout{0, 71} : SmemLayout{0, 63};
    case 60: return real_bytes == 4 ? SmemLayout{5, 61} : SmemLayout{2, 75};
    case 63: return real_bytes == 4 ? SmemLayout{4, 73} : SmemLayout{5, 65};
    case 64: return real_bytes == 4 ? SmemLayout{2, 87} : SmemLayout{3, 71};
    case 70: return real_bytes == 4 ? SmemLayout{0, 77} : SmemLayout{0, 70};
    case 72: return real_bytes == 4 ? SmemLayout{0, 73} : SmemLayout{3, 81};
    case 75: return real_bytes == 4 ? SmemLayout{0, 85} : SmemLayout{0, 75};
    case 80: return real_bytes == 4 ? SmemLayout{0, 85} : SmemLayout{2, 105};
    case 81: return real_bytes == 4 ? SmemLayout{0, 89} : SmemLayout{0, 83};
    case 84: return real_bytes == 4 ? SmemLayout{2, 105} : SmemLayout{0, 85};
    case 90: return real_bytes == 4 ? SmemLayout{0, 105} : SmemLayout{0, 91};
    case 96: return real_bytes == 4 ? SmemLayout{0, 97} : SmemLayout{2, 126};
    case 98: return real_bytes == 4 ? SmemLayout{0, 103} : SmemLayout{5, 102};
    case 100: return real_bytes == 4 ? SmemLayout{2, 125} : SmemLayout{2, 125};
    case 105: return real_bytes == 4 ? SmemLayout{0, 119} : SmemLayout{0, 107};
    case 108: return real_bytes == 4 ? SmemLayout{0, 121} : SmemLayout{0, 109};
    case 112: return real_bytes == 4 ? SmemLayout{4, 119} : SmemLayout{3, 132};
    case 120: return real_bytes == 4 ? SmemLayout{5, 138} : SmemLayout{3, 135};
    case 125: return real_bytes == 4 ? SmemLayout{0, 137} : SmemLayout{0, 125};
    case 126: return real_bytes == 4 ? SmemLayout{0, 137} : SmemLayout{5, 130};
    case 128: return real_bytes == 4 ? SmemLayout{4, 141} : SmemLayout{4, 135};
    case 135: return real_bytes == 4 ? SmemLayout{0, 137} : SmemLayout{0, 141};
    case 140: return real_bytes == 4 ? SmemLayout{5, 154} : SmemLayout{0, 140};
    case 144: return real_bytes == 4 ? SmemLayout{3, 162} : SmemLayout{5, 148};
    case 147: return real_bytes == 4 ? SmemLayout{0, 149} : SmemLayout{0, 149};
    case 150: return real_bytes == 4 ? SmemLayout{5, 154} : SmemLayout{0, 150};
    case 160: return real_bytes == 4 ? SmemLayout{0, 165} : SmemLayout{2, 201};
    case 162: return real_bytes == 4 ? SmemLayout{0, 162} : SmemLayout{2, 203};
    case 168: return real_bytes == 4 ? SmemLayout{3, 189} : SmemLayout{3, 189};
    case 175: return real_bytes == 4 ? SmemLayout{0, 179} : SmemLayout{0, 179};
    case 180: return real_bytes == 4 ? SmemLayout{2, 225} : SmemLayout{5, 190};
    case 189: return real_bytes == 4 ? SmemLayout{0, 203} : SmemLayout{0, 191};
    case 192: return real_bytes == 4 ? SmemLayout{2, 239} : SmemLayout{3, 215};
    case 196: return real_bytes == 4 ? SmemLayout{5, 206} : SmemLayout{2, 251};
    case 200: return real_bytes == 4 ? SmemLayout{4, 218} : SmemLayout{3, 225};
    case 210: return real_bytes == 4 ? SmemLayout{4, 238} : SmemLayout{0, 211};
    case 216: return real_bytes == 4 ? SmemLayout{0, 228} : SmemLayout{2, 269};
    case 224: return real_bytes == 4 ? SmemLayout{0, 238} : SmemLayout{4, 238};
    case 225: return real_bytes == 4 ? SmemLayout{0, 239} : SmemLayout{0, 225};
    case 240: return real_bytes == 4 ? SmemLayout{0, 255} : SmemLayout{0, 246};
    case 243: return real_bytes == 4 ? SmemLayout{0, 251} : SmemLayout{0, 249};
    case 245: return real_bytes == 4 ? SmemLayout{0, 259} : SmemLayout{0, 251};
    case 250: return real_bytes == 4 ? SmemLayout{0, 258} : SmemLayout{0, 250};
    case 252: return real_bytes == 4 ? SmemLayout{0, 266} : SmemLayout{5, 259};
    case 256: return real_bytes == 4 ? SmemLayout{4, 282} : SmemLayout{5, 263};
    case 270: return real_bytes == 4 ? SmemLayout{0, 278} : SmemLayout{0, 274};
    case 280: return real_bytes == 4 ? SmemLayout{0, 294} : SmemLayout{3, 315};
    case 288: return real_bytes == 4 ? SmemLayout{5, 302} : SmemLayout{3, 324};
    case 294: return real_bytes == 4 ? SmemLayout{0, 298} : SmemLayout{5, 307};
    case 300: return real_bytes == 4 ? SmemLayout{0, 300} : SmemLayout{0, 300};
    case 315: return real_bytes == 4 ? SmemLayout{0, 317} : SmemLayout{0, 321};
    case 320: return real_bytes == 4 ? SmemLayout{0, 334} : SmemLayout{3, 365};
    case 324: return real_bytes == 4 ? SmemLayout{0, 324} : SmemLayout{2, 410};
    case 336: return real_bytes == 4 ? SmemLayout{5, 348} : SmemLayout{3, 378};
    case 343: return real_bytes == 4 ? SmemLayout{5, 354} : SmemLayout{0, 345};
    case 350: return real_bytes == 4 ? SmemLayout{0, 350} : SmemLayout{0, 350};
    case 360: return real_bytes == 4 ? SmemLayout{0, 365} : SmemLayout{5, 371};
    case 375: return real_bytes == 4 ? SmemLayout{0, 379} : SmemLayout{0, 379};
    case 378: return real_bytes == 4 ? SmemLayout{0, 378} : SmemLayout{2, 478};
    case 384: return real_bytes == 4 ? SmemLayout{5, 398} : SmemLayout{3, 431};
    case 392: return real_bytes == 4 ? SmemLayout{0, 392} : SmemLayout{0, 393};
    case 400: return real_bytes == 4 ? SmemLayout{4, 425} : SmemLayout{2, 500};
    case 405: return real_bytes == 4 ? SmemLayout{0, 413} : SmemLayout{0, 407};
    case 420: return real_bytes == 4 ? SmemLayout{0, 420} : SmemLayout{2, 525};
    case 432: return real_bytes == 4 ? SmemLayout{4, 459} : SmemLayout{3, 486};
    case 441: return real_bytes == 4 ? SmemLayout{0, 452} : SmemLayout{0, 447};
    case 448: return real_bytes == 4 ? SmemLayout{0, 456} : SmemLayout{0, 449};
    case 450: return real_bytes == 4 ? SmemLayout{0, 461} : SmemLayout{0, 450};
    case 480: return real_bytes == 4 ? SmemLayout{4, 524} : SmemLayout{3, 540};
    case 486: return real_bytes == 4 ? SmemLayout{0, 486} : SmemLayout{2, 612};
    case 490: return real_bytes == 4 ? SmemLayout{0, 502} : SmemLayout{2, 612};
    case 500: return real_bytes == 4 ? SmemLayout{0, 500} : SmemLayout{2, 629};
    case 504: return real_bytes == 4 ? SmemLayout{4, 548} : SmemLayout{5, 519};
    case 512: return real_bytes == 4 ? SmemLayout{4, 548} : SmemLayout{5, 527};
    case 770: return real_bytes == 4 ? SmemLayout{0, 781} : SmemLayout{0, 774};
    default: return SmemLayout{3, N + N / 8 + 1};
  }
}

}  // namespace pb
