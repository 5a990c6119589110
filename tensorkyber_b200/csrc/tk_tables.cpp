// tk_tables.cpp -- host matrix builder: derives the four stage matrices of the
// ML-KEM NTT by probing a modular restatement of the butterfly layers with unit
// vectors (the construction of ntt_bench/ntt_kernels.cuh:831-925), then packs
// them into 7-bit INT8 limb fragments in mma.sync register order.
#include "tk_tables.h"

#include <string.h>

namespace tk {
namespace {

int64_t modq(int64_t v) {
  v %= kQ;
  return v < 0 ? v + kQ : v;
}

unsigned brv7(unsigned x) {
  unsigned r = 0;
  for (int b = 0; b < 7; b++) r |= ((x >> b) & 1u) << (6 - b);
  return r;
}

// Twiddle k of the reference table (ntt_bench/ref/ntt.c:39-56) is
// 2^16 * 17^brv7(k) mod q; its Montgomery product fqmul(z, v) = z * 2^-16 * v,
// so in plain modular arithmetic the butterfly constant is 17^brv7(k).
struct Twiddles {
  int64_t w[128];
  Twiddles() {
    for (unsigned k = 0; k < 128; k++) {
      int64_t acc = 1;
      for (unsigned e = 0; e < brv7(k); e++) acc = acc * 17 % kQ;
      w[k] = acc;
    }
  }
};
const Twiddles& tw() {
  static const Twiddles t;
  return t;
}

// Forward Cooley-Tukey layers with len in [len_lo, len_hi] (ref/ntt.c:80-95):
// the twiddle index of (len, start) is 128/len + start/(2 len).
void fwd_layers(int64_t r[256], unsigned len_hi, unsigned len_lo) {
  for (unsigned len = len_hi; len >= len_lo; len >>= 1)
    for (unsigned start = 0; start < 256; start += 2 * len) {
      const int64_t z = tw().w[128 / len + start / (2 * len)];
      for (unsigned j = start; j < start + len; j++) {
        const int64_t t = z * r[j + len] % kQ;
        const int64_t a = r[j];
        r[j] = modq(a + t);
        r[j + len] = modq(a - t);
      }
    }
}

// Inverse Gentleman-Sande layers with len in [len_lo, len_hi] (ref/ntt.c:106-122):
// twiddle index 256/len - 1 - start/(2 len) (the k-- walk from 127).
void inv_layers(int64_t r[256], unsigned len_lo, unsigned len_hi) {
  for (unsigned len = len_lo; len <= len_hi; len <<= 1)
    for (unsigned start = 0; start < 256; start += 2 * len) {
      const int64_t z = tw().w[256 / len - 1 - start / (2 * len)];
      for (unsigned j = start; j < start + len; j++) {
        const int64_t a = r[j], b = r[j + len];
        r[j] = modq(a + b);
        r[j + len] = modq(z * modq(b - a));
      }
    }
}

// The final fqmul(r, 1441) of ref/ntt.c:124-125 multiplies by
// 1441 * 2^-16 = 2^16 / 128 = 512 (mod q).
constexpr int64_t kInvScale = 512;

uint8_t limb(int64_t v, int g) { return (uint8_t)(g ? (v >> 7) : (v & 127)); }

// c * 256^byte mod q: the constant that byte `byte` of a data word carries.
int64_t byte_weighted(int64_t c, int byte) {
  int64_t v = modq(c);
  for (int j = 0; j < byte; j++) v = v * 256 % kQ;
  return v;
}

}  // namespace

void build_pair_roots(int32_t z[128]) {
  for (int t = 0; t < 128; t++) {
    const int64_t w = tw().w[64 + t / 2];
    z[t] = (int32_t)((t & 1) ? modq(-w) : w);
  }
}

void build_pair_constants(int32_t zr[128]) {
  const int64_t rinv = 169;  // 2^-16 mod q
  build_pair_roots(zr);
  for (int t = 0; t < 128; t++) zr[t] = (int32_t)(zr[t] * rinv % kQ);
}

void scale_inverse(Matrices* M, int64_t f) {
  for (int i = 0; i < 16; i++)
    for (int m = 0; m < 16; m++) M->minv[i][m] = (int16_t)modq(M->minv[i][m] * f);
}

void build_matrices(Matrices* M) {
  int64_t v[256];
  for (int m = 0; m < 16; m++) {
    memset(v, 0, sizeof(v));
    v[16 * m] = 1;
    fwd_layers(v, 128, 16);
    for (int i = 0; i < 16; i++) M->m1[i][m] = (int16_t)v[16 * i];

    memset(v, 0, sizeof(v));
    v[16 * m] = 1;
    inv_layers(v, 16, 128);
    for (int i = 0; i < 16; i++) M->minv[i][m] = (int16_t)modq(v[16 * i] * kInvScale);
  }
  for (int b = 0; b < 16; b++)
    for (int c = 0; c < 16; c++) {
      memset(v, 0, sizeof(v));
      v[16 * b + c] = 1;
      fwd_layers(v, 8, 2);
      for (int co = 0; co < 16; co++) M->m2[b][co][c] = (int16_t)v[16 * b + co];

      memset(v, 0, sizeof(v));
      v[16 * b + c] = 1;
      inv_layers(v, 2, 8);
      for (int co = 0; co < 16; co++) M->ma[b][co][c] = (int16_t)v[16 * b + co];
    }
}

// m16n8k32 A fragment, 8-bit: reg j byte e holds A[row][col] with
// row = lane/4 (+8 for j odd), col = 4*(lane%4) + e (+16 for j >= 2).
template <class F>
static void pack_a_k32(F value, uint32_t out[32][4]) {
  for (int lane = 0; lane < 32; lane++)
    for (int j = 0; j < 4; j++) {
      uint32_t w = 0;
      for (int e = 0; e < 4; e++) {
        const int row = (lane >> 2) + ((j & 1) ? 8 : 0);
        const int col = 4 * (lane & 3) + e + ((j & 2) ? 16 : 0);
        w |= (uint32_t)value(row, col) << (8 * e);
      }
      out[lane][j] = w;
    }
}

// m16n8k16 A fragment, 8-bit: reg j byte e holds A[lane/4 + 8j][4*(lane%4) + e].
template <class F>
static void pack_a_k16(F value, uint32_t out[32][2]) {
  for (int lane = 0; lane < 32; lane++)
    for (int j = 0; j < 2; j++) {
      uint32_t w = 0;
      for (int e = 0; e < 4; e++)
        w |= (uint32_t)value((lane >> 2) + 8 * j, 4 * (lane & 3) + e) << (8 * e);
      out[lane][j] = w;
    }
}

void build_fwd_frags(const Matrices& M, FwdFrags* F) {
  for (int g = 0; g < 2; g++)
    pack_a_k32([&](int i, int k) { return limb(byte_weighted(M.m1[i][k >> 1], k & 1), g); },
               F->s1[g]);
  int32_t corr[16];
  for (int i = 0; i < 16; i++) {
    int64_t rs = 0;
    for (int m = 0; m < 16; m++) rs += M.m1[i][m];
    corr[i] = (int32_t)modq(-32768 * rs);
  }
  for (int lane = 0; lane < 32; lane++) {
    F->c1[lane][0] = corr[lane >> 2];
    F->c1[lane][1] = corr[(lane >> 2) + 8];
  }
  for (int b = 0; b < 16; b++)
    for (int s = 0; s < 2; s++)
      pack_a_k16(
          [&](int r, int k) {
            const int co = 2 * (r & 7) + s;
            const int c = 2 * fwd_slot_e(k >> 1) + s;
            return limb(byte_weighted(M.m2[b][co][c], k & 1), r >> 3);
          },
          F->s2[b][s]);
  for (int b = 0; b < 16; b++)
    for (int s = 0; s < 2; s++)
      pack_a_k32(
          [&](int r, int k) {
            const int co = 2 * (r & 7) + s;
            const int c = 2 * fwd_slot_e(k >> 2) + s;
            return limb(byte_weighted(M.m2[b][co][c], k & 3), r >> 3);
          },
          F->s2w[b][s]);
  // single-limb stage 1: two accumulator groups (lo / hi limb), rows 0..15
  // on the two A register halves of m16n8k16
  for (int g = 0; g < 2; g++)
    pack_a_k16([&](int i, int k) { return limb(M.m1[i][basic_k_block(k)], g); }, F->s1b[g]);
  for (int i = 0; i < 16; i++) {
    int64_t rs = 0;
    for (int m = 0; m < 16; m++) rs += M.m1[i][m];
    corr[i] = (int32_t)modq(-128 * rs);
  }
  for (int lane = 0; lane < 32; lane++) {
    F->c1b[lane][0] = corr[lane >> 2];
    F->c1b[lane][1] = corr[(lane >> 2) + 8];
  }
}

int basic_k_block(int k) {
  const int t = k >> 2, j = k & 3;
  return j < 2 ? 2 * t + j : 8 + 2 * t + (j - 2);
}

void build_inv_frags(const Matrices& M, InvFrags* F) {
  for (int b = 0; b < 16; b++)
    for (int s = 0; s < 2; s++) {
      pack_a_k16(
          [&](int r, int k) {
            const int co = 2 * (r & 7) + s;
            const int c = 2 * fwd_slot_e(k >> 1) + s;
            return limb(byte_weighted(M.ma[b][co][c], k & 1), r >> 3);
          },
          F->sa[b][s]);
      for (int lane = 0; lane < 32; lane++) {
        const int co = 2 * (lane >> 2) + s;
        int64_t rs = 0;
        for (int c = 0; c < 16; c++) rs += M.ma[b][co][c];
        F->ca[b][s][lane] = (int32_t)modq(-32768 * rs);
      }
    }
  for (int g = 0; g < 2; g++)
    pack_a_k32([&](int i, int k) { return limb(byte_weighted(M.minv[i][k >> 1], k & 1), g); },
               F->sb[g]);
  for (int g = 0; g < 2; g++)
    for (int j = 0; j < 2; j++)
      pack_a_k32(
          [&](int i, int k) { return limb(byte_weighted(M.minv[i][8 * j + (k >> 2)], k & 3), g); },
          F->sbw[g][j]);
  // stage B init that cancels stage A's bias offset 32768 * rowsum(MA[m][c])
  int64_t off[16][16];
  for (int m = 0; m < 16; m++)
    for (int c = 0; c < 16; c++) {
      int64_t rs = 0;
      for (int j = 0; j < 16; j++) rs += M.ma[m][c][j];
      off[m][c] = modq(32768 * rs);
    }
  auto init = [&](int i, int c) {
    int64_t v = 0;
    for (int m = 0; m < 16; m++) v += (int64_t)M.minv[i][m] * off[m][c];
    return (int32_t)modq(-v);
  };
  for (int lane = 0; lane < 32; lane++)
    for (int t = 0; t < 2; t++) {
      const int i = lane >> 2, c = 8 * t + 2 * (lane & 3);
      F->cbz[lane][t][0] = init(i, c);
      F->cbz[lane][t][1] = init(i, c + 1);
      F->cbz[lane][t][2] = init(i + 8, c);
      F->cbz[lane][t][3] = init(i + 8, c + 1);
    }
}

void build_tc5_tables(const Matrices& M, uint8_t* out) {
  memset(out, 0, kTc5TableBytes);
  auto put = [&](int tile, int n, int k, int64_t v) {
    out[tile * kTc5TileBytes + tc5_tile_offset(n, k)] = (uint8_t)v;
  };
  for (int o = 0; o < 16; o++)
    for (int g = 0; g < 2; g++)
      for (int j = 0; j < 16; j++)
        for (int b = 0; b < 2; b++) {
          // inverse stage A, every block m: input coefficient j
          for (int m = 0; m < 16; m++) {
            if (b == 0) put(2 * m, o + 16 * g, 2 * j, limb(M.ma[m][o][j], g));
            else put(2 * m + 1, o + 16 * g, 2 * j + 1, limb(byte_weighted(M.ma[m][o][j], 1), g));
          }
          // forward stage 1: input block j, byte b (unsigned low / signed high)
          put(34 + b, o + 16 * g, 2 * j + b, limb(byte_weighted(M.m1[o][j], b), g));
        }
  // second stages: four bytes of an int32 sum per input, two K steps of 8
  for (int o = 0; o < 16; o++)
    for (int g = 0; g < 2; g++)
      for (int j = 0; j < 16; j++)
        for (int t = 0; t < 4; t++) {
          const int h = j >> 3, k = 4 * (j & 7) + t;
          put(32 + h, o + 16 * g, k, limb(byte_weighted(M.minv[o][j], t), g));
          for (int i = 0; i < 16; i++)
            put(36 + 2 * i + h, o + 16 * g, k, limb(byte_weighted(M.m2[i][o][j], t), g));
        }
}

}  // namespace tk
