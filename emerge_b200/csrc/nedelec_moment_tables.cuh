// GENERATED by gen_tables.py -- do not edit.
// Quadrature-moment form of the Nedelec-2 (Volakis mixed) element integrals:
// entries = sum over tensor terms T[a][b] * (sum_alpha c_alpha * mu[alpha]),
// mu[alpha] = sum_q w_q L_q^alpha over the 11 KEAST4 points.
#pragma once
namespace emg_mtables {
constexpr int kNumMoments = 70;
template <class R>
__device__ __forceinline__ void emg_moments(const R L[4], R w, R mu[kNumMoments]) {
  const R m0 = w;
  mu[0] += m0;
  const R m1 = m0 * L[0];
  mu[1] += m1;
  const R m2 = m0 * L[1];
  mu[2] += m2;
  const R m3 = m0 * L[2];
  mu[3] += m3;
  const R m4 = m0 * L[3];
  mu[4] += m4;
  const R m5 = m1 * L[0];
  mu[5] += m5;
  const R m6 = m1 * L[1];
  mu[6] += m6;
  const R m7 = m1 * L[2];
  mu[7] += m7;
  const R m8 = m1 * L[3];
  mu[8] += m8;
  const R m9 = m2 * L[1];
  mu[9] += m9;
  const R m10 = m2 * L[2];
  mu[10] += m10;
  const R m11 = m2 * L[3];
  mu[11] += m11;
  const R m12 = m3 * L[2];
  mu[12] += m12;
  const R m13 = m3 * L[3];
  mu[13] += m13;
  const R m14 = m4 * L[3];
  mu[14] += m14;
  const R m15 = m5 * L[0];
  mu[15] += m15;
  const R m16 = m5 * L[1];
  mu[16] += m16;
  const R m17 = m5 * L[2];
  mu[17] += m17;
  const R m18 = m5 * L[3];
  mu[18] += m18;
  const R m19 = m6 * L[1];
  mu[19] += m19;
  const R m20 = m6 * L[2];
  mu[20] += m20;
  const R m21 = m6 * L[3];
  mu[21] += m21;
  const R m22 = m7 * L[2];
  mu[22] += m22;
  const R m23 = m7 * L[3];
  mu[23] += m23;
  const R m24 = m8 * L[3];
  mu[24] += m24;
  const R m25 = m9 * L[1];
  mu[25] += m25;
  const R m26 = m9 * L[2];
  mu[26] += m26;
  const R m27 = m9 * L[3];
  mu[27] += m27;
  const R m28 = m10 * L[2];
  mu[28] += m28;
  const R m29 = m10 * L[3];
  mu[29] += m29;
  const R m30 = m11 * L[3];
  mu[30] += m30;
  const R m31 = m12 * L[2];
  mu[31] += m31;
  const R m32 = m12 * L[3];
  mu[32] += m32;
  const R m33 = m13 * L[3];
  mu[33] += m33;
  const R m34 = m14 * L[3];
  mu[34] += m34;
  const R m35 = m15 * L[0];
  mu[35] += m35;
  const R m36 = m15 * L[1];
  mu[36] += m36;
  const R m37 = m15 * L[2];
  mu[37] += m37;
  const R m38 = m15 * L[3];
  mu[38] += m38;
  const R m39 = m16 * L[1];
  mu[39] += m39;
  const R m40 = m16 * L[2];
  mu[40] += m40;
  const R m41 = m16 * L[3];
  mu[41] += m41;
  const R m42 = m17 * L[2];
  mu[42] += m42;
  const R m43 = m17 * L[3];
  mu[43] += m43;
  const R m44 = m18 * L[3];
  mu[44] += m44;
  const R m45 = m19 * L[1];
  mu[45] += m45;
  const R m46 = m19 * L[2];
  mu[46] += m46;
  const R m47 = m19 * L[3];
  mu[47] += m47;
  const R m48 = m20 * L[2];
  mu[48] += m48;
  const R m49 = m20 * L[3];
  mu[49] += m49;
  const R m50 = m21 * L[3];
  mu[50] += m50;
  const R m51 = m22 * L[2];
  mu[51] += m51;
  const R m52 = m22 * L[3];
  mu[52] += m52;
  const R m53 = m23 * L[3];
  mu[53] += m53;
  const R m54 = m24 * L[3];
  mu[54] += m54;
  const R m55 = m25 * L[1];
  mu[55] += m55;
  const R m56 = m25 * L[2];
  mu[56] += m56;
  const R m57 = m25 * L[3];
  mu[57] += m57;
  const R m58 = m26 * L[2];
  mu[58] += m58;
  const R m59 = m26 * L[3];
  mu[59] += m59;
  const R m60 = m27 * L[3];
  mu[60] += m60;
  const R m61 = m28 * L[2];
  mu[61] += m61;
  const R m62 = m28 * L[3];
  mu[62] += m62;
  const R m63 = m29 * L[3];
  mu[63] += m63;
  const R m64 = m30 * L[3];
  mu[64] += m64;
  const R m65 = m31 * L[2];
  mu[65] += m65;
  const R m66 = m31 * L[3];
  mu[66] += m66;
  const R m67 = m32 * L[3];
  mu[67] += m67;
  const R m68 = m33 * L[3];
  mu[68] += m68;
  const R m69 = m34 * L[3];
  mu[69] += m69;
}
template <int f, int s> struct MPair;
template <> struct MPair<0, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[9])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[6])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[6])); emg_mac(acc, G[1][1], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<0, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[10])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[6])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[7])); emg_mac(acc, G[1][2], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<0, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[11])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[6])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[8])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<0, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[10])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[9])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[7])); emg_mac(acc, G[1][2], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<0, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[11])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[9])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<0, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[11])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[10])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<0, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[25])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<0, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[28])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[20])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<0, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[30])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[21])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<0, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[28])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[25]), 1.0, mu[26])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<0, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[27]), -1.0, mu[30])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[25]), 1.0, mu[27])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<0, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[30])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[28]), 1.0, mu[29])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<0, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[0][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[0][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[20])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[19])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[17])); emg_mac(acc, G[1][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<0, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[0][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[21])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[19])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[18])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<0, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[0][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[21])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[18])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<0, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[0][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[27])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[26])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<0, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[0][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[0][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[26])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[19])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[1][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<0, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[0][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[27])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[19])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<0, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[0][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[1][0], emg_mul(-1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<0, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[0][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[26])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<1, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[10])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[6])); emg_mac(acc, G[2][1], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<1, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[12])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<1, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[8])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<1, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[12])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<1, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[13])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<1, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[13])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[12])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<1, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[26])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[20])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<1, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[31])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<1, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[33])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[23])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<1, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[31])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<1, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[33])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[29])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<1, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[32]), -1.0, mu[33])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[31]), 1.0, mu[32])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<1, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[1][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[22])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[17])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<1, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[1][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[18])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<1, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[23])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[22])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[18])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<1, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[28])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<1, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[28])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<1, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[1][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<1, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[1][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[32])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[22])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[23])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<1, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[1][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[32])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[28])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<2, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[11])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[6])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<2, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[7])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<2, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[14])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[5])); }
};
template <> struct MPair<2, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[13])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[7])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<2, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[14])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<2, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[14])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<2, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<2, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<2, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<2, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<2, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<2, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<2, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[2][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[17])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<2, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[24])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<2, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[24])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<2, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[30])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<2, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[2][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<2, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[30])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<2, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[33])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<2, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[33])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<3, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[10])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[9])); emg_mac(acc, G[2][1], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<3, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[12])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<3, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[13])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[7])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[11])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<3, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[12])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[9])); }
};
template <> struct MPair<3, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[13])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[10])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[11])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[9])); }
};
template <> struct MPair<3, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[13])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[12])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[11])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[10])); }
};
template <> struct MPair<3, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[26])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[20])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[19]), 1.0, mu[25])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[19])); }
};
template <> struct MPair<3, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[31])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[28])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[20])); }
};
template <> struct MPair<3, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[33])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[23])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[30])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[21])); }
};
template <> struct MPair<3, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[31])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[26])); }
};
template <> struct MPair<3, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[33])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[29])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[27])); }
};
template <> struct MPair<3, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[32]), -1.0, mu[33])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[31]), 1.0, mu[32])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[30])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[29])); }
};
template <> struct MPair<3, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[22])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<3, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<3, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[3][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[22])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<3, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[3][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[29])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[28])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[27])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<3, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[3][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[28])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[26])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<3, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[3][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[27])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<3, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[3][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[32])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[22])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[29])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<3, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[3][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[32])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[28])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[29])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<4, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[11])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[9])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<4, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[13])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[10])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<4, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[14])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[6])); }
};
template <> struct MPair<4, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[13])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[10])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[9])); }
};
template <> struct MPair<4, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[14])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[9])); }
};
template <> struct MPair<4, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[14])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[10])); }
};
template <> struct MPair<4, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[19]), 1.0, mu[25])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[19])); }
};
template <> struct MPair<4, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[28])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[20])); }
};
template <> struct MPair<4, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[21])); }
};
template <> struct MPair<4, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[26])); }
};
template <> struct MPair<4, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[27])); }
};
template <> struct MPair<4, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[29])); }
};
template <> struct MPair<4, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<4, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[24])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<4, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[24])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<4, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[30])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<4, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[4][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[26])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<4, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[30])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<4, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[33])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<4, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[33])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<5, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[11])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[10])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<5, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[13])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[12])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<5, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][2], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[14])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[8])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[7])); }
};
template <> struct MPair<5, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[13])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[12])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[10])); }
};
template <> struct MPair<5, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][4], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[14])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[11])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[10])); }
};
template <> struct MPair<5, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][5], emg_mul(4.0, mu[0])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[14])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[13])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[12])); }
};
template <> struct MPair<5, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[26])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[20])); }
};
template <> struct MPair<5, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[22]), 1.0, mu[31])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[22])); }
};
template <> struct MPair<5, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[23])); }
};
template <> struct MPair<5, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[28]), 1.0, mu[31])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[28])); }
};
template <> struct MPair<5, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[29])); }
};
template <> struct MPair<5, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[31]), -1.0, mu[32])); }
};
template <> struct MPair<5, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[5][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[22])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<5, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[24])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<5, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[24])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[22])); }
};
template <> struct MPair<5, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[30])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[28])); }
};
template <> struct MPair<5, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[28])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<5, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[30])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<5, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[33])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[32])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[22])); }
};
template <> struct MPair<5, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[33])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[32])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[28])); }
};
template <> struct MPair<6, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[25])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<6, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[26])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[20])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<6, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[19])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[16])); }
};
template <> struct MPair<6, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[26])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[19]), 1.0, mu[25])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[20])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[19])); }
};
template <> struct MPair<6, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[19]), 1.0, mu[25])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[19])); }
};
template <> struct MPair<6, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[27])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[26])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[21])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[20])); }
};
template <> struct MPair<6, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_fma(emg_mul(9.0, mu[5]), -18.0, mu[6]), 9.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_mul(1.0, mu[39]), -2.0, mu[45]), 1.0, mu[55])); emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 2.0, mu[39]), -1.0, mu[45])); emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 2.0, mu[39]), -1.0, mu[45])); emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_mul(1.0, mu[35]), -2.0, mu[36]), 1.0, mu[39])); }
};
template <> struct MPair<6, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[6]), -9.0, mu[7]), 9.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46]), -1.0, mu[48]), 1.0, mu[58])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 1.0, mu[39]), 1.0, mu[40]), -1.0, mu[46])); emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[40]), 1.0, mu[42]), -1.0, mu[48])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[36]), -1.0, mu[37]), 1.0, mu[40])); }
};
template <> struct MPair<6, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[6]), -9.0, mu[8]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47]), -1.0, mu[50]), 1.0, mu[60])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 1.0, mu[39]), 1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41]), 1.0, mu[44]), -1.0, mu[50])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[36]), -1.0, mu[38]), 1.0, mu[41])); }
};
template <> struct MPair<6, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[9]), 9.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48]), -1.0, mu[56]), 1.0, mu[58])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[45]), 1.0, mu[46]), 1.0, mu[55]), -1.0, mu[56])); emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[46]), -1.0, mu[48])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[45]), 1.0, mu[46])); }
};
template <> struct MPair<6, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[9]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[50]), -1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[45]), 1.0, mu[47]), 1.0, mu[55]), -1.0, mu[57])); emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[47]), -1.0, mu[50])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[45]), 1.0, mu[47])); }
};
template <> struct MPair<6, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[10]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[50]), -1.0, mu[59]), 1.0, mu[60])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[49]), 1.0, mu[58]), -1.0, mu[59])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[49]), -1.0, mu[50])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[48]), 1.0, mu[49])); }
};
template <> struct MPair<6, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[10])); emg_mac(acc, H[0][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); emg_mac(acc, H[0][3], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[40])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<6, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[0][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); emg_mac(acc, H[0][4], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<6, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[0][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[0][5], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[40])); }
};
template <> struct MPair<6, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[0][4], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[0][5], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[57])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[56])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[47])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); }
};
template <> struct MPair<6, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[0][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); emg_mac(acc, H[0][3], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[56])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<6, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[0][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); emg_mac(acc, H[0][4], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[57])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[47])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<6, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[0][2], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[10])); emg_mac(acc, H[0][5], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[59])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[1][0], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[49])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[40])); }
};
template <> struct MPair<6, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[0][4], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[10])); emg_mac(acc, H[0][5], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[59])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[56])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[49])); emg_mac(acc, G[1][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); }
};
template <> struct MPair<7, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[20]), -1.0, mu[28])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[20])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<7, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[31])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<7, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[17])); }
};
template <> struct MPair<7, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[31])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[22])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[20])); }
};
template <> struct MPair<7, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[20])); }
};
template <> struct MPair<7, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[32])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[22]), 1.0, mu[31])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[23])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[22])); }
};
template <> struct MPair<7, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[6]), -9.0, mu[7]), 9.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46]), -1.0, mu[48]), 1.0, mu[58])); emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[40]), 1.0, mu[42]), -1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 1.0, mu[39]), 1.0, mu[40]), -1.0, mu[46])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[36]), -1.0, mu[37]), 1.0, mu[40])); }
};
template <> struct MPair<7, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_fma(emg_mul(9.0, mu[5]), -18.0, mu[7]), 9.0, mu[12])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_mul(1.0, mu[42]), -2.0, mu[51]), 1.0, mu[65])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 2.0, mu[42]), -1.0, mu[51])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 2.0, mu[42]), -1.0, mu[51])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_mul(1.0, mu[35]), -2.0, mu[37]), 1.0, mu[42])); }
};
template <> struct MPair<7, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[7]), -9.0, mu[8]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52]), -1.0, mu[53]), 1.0, mu[67])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[42]), 1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43]), 1.0, mu[44]), -1.0, mu[53])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[37]), -1.0, mu[38]), 1.0, mu[43])); }
};
template <> struct MPair<7, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[10]), 9.0, mu[12])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[51]), -1.0, mu[61]), 1.0, mu[65])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48]), 1.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[48]), -1.0, mu[51])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[46]), 1.0, mu[48])); }
};
template <> struct MPair<7, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[10]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[53]), -1.0, mu[62]), 1.0, mu[67])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[49]), 1.0, mu[58]), -1.0, mu[62])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[49]), -1.0, mu[53])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[46]), 1.0, mu[49])); }
};
template <> struct MPair<7, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[12]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[53]), -1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[51]), 1.0, mu[52]), 1.0, mu[65]), -1.0, mu[66])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[52]), -1.0, mu[53])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[51]), 1.0, mu[52])); }
};
template <> struct MPair<7, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[12])); emg_mac(acc, H[1][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); emg_mac(acc, H[1][3], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[51])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[42])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<7, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); emg_mac(acc, H[1][4], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<7, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[1][5], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[42]), 1.0, mu[51])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[42])); }
};
template <> struct MPair<7, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[1][4], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[1][5], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[62])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[61])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[49])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[48])); }
};
template <> struct MPair<7, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[1][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); emg_mac(acc, H[1][3], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[61])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<7, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); emg_mac(acc, H[1][4], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[62])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[49])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<7, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[12])); emg_mac(acc, H[1][5], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[66])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[42]), 1.0, mu[51])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[52])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[42])); }
};
template <> struct MPair<7, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[1][4], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[12])); emg_mac(acc, H[1][5], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[66])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[61])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[52])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[48])); }
};
template <> struct MPair<8, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[21]), -1.0, mu[30])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[16]), 1.0, mu[21])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<8, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[33])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[23])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<8, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[15]), -1.0, mu[18])); }
};
template <> struct MPair<8, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[23]), -1.0, mu[33])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[17]), 1.0, mu[23])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[21])); }
};
template <> struct MPair<8, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[16]), -1.0, mu[21])); }
};
template <> struct MPair<8, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[1]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[24]), -1.0, mu[34])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[18]), 1.0, mu[24])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[17]), -1.0, mu[23])); }
};
template <> struct MPair<8, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[6]), -9.0, mu[8]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47]), -1.0, mu[50]), 1.0, mu[60])); emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41]), 1.0, mu[44]), -1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[36]), 1.0, mu[39]), 1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[36]), -1.0, mu[38]), 1.0, mu[41])); }
};
template <> struct MPair<8, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[5]), -9.0, mu[7]), -9.0, mu[8]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52]), -1.0, mu[53]), 1.0, mu[67])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43]), 1.0, mu[44]), -1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[42]), 1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[35]), -1.0, mu[37]), -1.0, mu[38]), 1.0, mu[43])); }
};
template <> struct MPair<8, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][2], emg_fma(emg_fma(emg_mul(9.0, mu[5]), -18.0, mu[8]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_fma(emg_mul(1.0, mu[44]), -2.0, mu[54]), 1.0, mu[69])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 2.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_mul(-1.0, mu[38]), 2.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_mul(1.0, mu[35]), -2.0, mu[38]), 1.0, mu[44])); }
};
template <> struct MPair<8, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[11]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52]), -1.0, mu[63]), 1.0, mu[67])); emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49]), 1.0, mu[60]), -1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[47]), 1.0, mu[49])); }
};
template <> struct MPair<8, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][4], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[11]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54]), -1.0, mu[64]), 1.0, mu[69])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50]), 1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[47]), 1.0, mu[50])); }
};
template <> struct MPair<8, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][5], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[13]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54]), -1.0, mu[68]), 1.0, mu[69])); emg_mac(acc, G[0][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53]), 1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[52]), 1.0, mu[53])); }
};
template <> struct MPair<8, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); emg_mac(acc, H[2][3], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[53])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[43])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<8, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[44])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<8, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[44])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[43])); }
};
template <> struct MPair<8, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[64])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[63])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[49])); }
};
template <> struct MPair<8, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); emg_mac(acc, H[2][3], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[63])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[49])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<8, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); emg_mac(acc, H[2][4], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[64])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<8, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[13])); emg_mac(acc, H[2][5], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[68])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[43])); }
};
template <> struct MPair<8, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[2][3], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[13])); emg_mac(acc, H[2][5], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[68])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[49])); }
};
template <> struct MPair<9, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[28])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[25]), 1.0, mu[26])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<9, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[31])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<9, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[20]), 1.0, mu[22])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[20])); }
};
template <> struct MPair<9, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[31])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[26])); }
};
template <> struct MPair<9, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[28])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[26])); }
};
template <> struct MPair<9, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[3])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[32])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[28]), 1.0, mu[31])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[29])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[28])); }
};
template <> struct MPair<9, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[9]), 9.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48]), -1.0, mu[56]), 1.0, mu[58])); emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[46]), -1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[45]), 1.0, mu[46]), 1.0, mu[55]), -1.0, mu[56])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[45]), 1.0, mu[46])); }
};
template <> struct MPair<9, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[10]), 9.0, mu[12])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[51]), -1.0, mu[61]), 1.0, mu[65])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[48]), -1.0, mu[51])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48]), 1.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[46]), 1.0, mu[48])); }
};
template <> struct MPair<9, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[7]), -9.0, mu[11]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52]), -1.0, mu[63]), 1.0, mu[67])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[42]), 1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49]), 1.0, mu[60]), -1.0, mu[63])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[40]), -1.0, mu[47]), 1.0, mu[49])); }
};
template <> struct MPair<9, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_fma(emg_mul(9.0, mu[9]), -18.0, mu[10]), 9.0, mu[12])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_mul(1.0, mu[58]), -2.0, mu[61]), 1.0, mu[65])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_mul(-1.0, mu[56]), 2.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_mul(-1.0, mu[56]), 2.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_mul(1.0, mu[55]), -2.0, mu[56]), 1.0, mu[58])); }
};
template <> struct MPair<9, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[9]), -9.0, mu[10]), -9.0, mu[11]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62]), -1.0, mu[63]), 1.0, mu[67])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[58]), 1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59]), 1.0, mu[60]), -1.0, mu[63])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[55]), -1.0, mu[56]), -1.0, mu[57]), 1.0, mu[59])); }
};
template <> struct MPair<9, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[10]), -9.0, mu[11]), -9.0, mu[12]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[63]), -1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[61]), 1.0, mu[62]), 1.0, mu[65]), -1.0, mu[66])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[60]), 1.0, mu[62]), -1.0, mu[63])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[59]), -1.0, mu[61]), 1.0, mu[62])); }
};
template <> struct MPair<9, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(-3.0, mu[10]), 3.0, mu[12])); emg_mac(acc, H[3][1], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); emg_mac(acc, H[3][3], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[51])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<9, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[3][2], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); emg_mac(acc, H[3][4], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<9, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[3][2], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[3][5], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[51])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48])); }
};
template <> struct MPair<9, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[3][4], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[3][5], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[58]), 1.0, mu[61])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[58])); }
};
template <> struct MPair<9, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[3][1], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); emg_mac(acc, H[3][3], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[58])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<9, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[3][2], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); emg_mac(acc, H[3][4], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<9, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[3][2], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[12])); emg_mac(acc, H[3][5], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[66])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[51])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[62])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48])); }
};
template <> struct MPair<9, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[3][4], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[12])); emg_mac(acc, H[3][5], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[66])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[58]), 1.0, mu[61])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[62])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[58])); }
};
template <> struct MPair<10, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[27]), -1.0, mu[30])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[25]), 1.0, mu[27])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<10, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[33])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[29])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<10, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[21]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[19]), -1.0, mu[21])); }
};
template <> struct MPair<10, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[33])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[26]), 1.0, mu[29])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[27])); }
};
template <> struct MPair<10, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[25]), -1.0, mu[27])); }
};
template <> struct MPair<10, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[2]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[30]), -1.0, mu[34])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[27]), 1.0, mu[30])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[26]), -1.0, mu[29])); }
};
template <> struct MPair<10, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[9]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[50]), -1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[47]), -1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[45]), 1.0, mu[47]), 1.0, mu[55]), -1.0, mu[57])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[45]), 1.0, mu[47])); }
};
template <> struct MPair<10, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[10]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[53]), -1.0, mu[62]), 1.0, mu[67])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[49]), -1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[49]), 1.0, mu[58]), -1.0, mu[62])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[46]), 1.0, mu[49])); }
};
template <> struct MPair<10, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][2], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[6]), -9.0, mu[8]), -9.0, mu[11]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54]), -1.0, mu[64]), 1.0, mu[69])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[44]), 1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50]), 1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[39]), -1.0, mu[41]), -1.0, mu[47]), 1.0, mu[50])); }
};
template <> struct MPair<10, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[9]), -9.0, mu[10]), -9.0, mu[11]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62]), -1.0, mu[63]), 1.0, mu[67])); emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59]), 1.0, mu[60]), -1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[58]), 1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[55]), -1.0, mu[56]), -1.0, mu[57]), 1.0, mu[59])); }
};
template <> struct MPair<10, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][4], emg_fma(emg_fma(emg_mul(9.0, mu[9]), -18.0, mu[11]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_fma(emg_mul(1.0, mu[60]), -2.0, mu[64]), 1.0, mu[69])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_mul(-1.0, mu[57]), 2.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_mul(-1.0, mu[57]), 2.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_mul(1.0, mu[55]), -2.0, mu[57]), 1.0, mu[60])); }
};
template <> struct MPair<10, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][5], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[10]), -9.0, mu[11]), -9.0, mu[13]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64]), -1.0, mu[68]), 1.0, mu[69])); emg_mac(acc, G[1][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63]), 1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[60]), 1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[59]), -1.0, mu[62]), 1.0, mu[63])); }
};
template <> struct MPair<10, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(-3.0, mu[10]), 3.0, mu[13])); emg_mac(acc, H[4][1], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); emg_mac(acc, H[4][3], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[53])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[49])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<10, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<10, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[53])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[49])); }
};
template <> struct MPair<10, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[4][4], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[59])); }
};
template <> struct MPair<10, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[4][1], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); emg_mac(acc, H[4][3], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[63])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[59])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<10, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][0], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); emg_mac(acc, H[4][4], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<10, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][1], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[13])); emg_mac(acc, H[4][5], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[68])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[49])); }
};
template <> struct MPair<10, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[4][3], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[13])); emg_mac(acc, H[4][5], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[68])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[59])); }
};
template <> struct MPair<11, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[29]), -1.0, mu[30])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[28]), 1.0, mu[29])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<11, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[32]), -1.0, mu[33])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[31]), 1.0, mu[32])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<11, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[23]), 1.0, mu[24])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[22]), -1.0, mu[23])); }
};
template <> struct MPair<11, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[32]), -1.0, mu[33])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[31]), 1.0, mu[32])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[29])); }
};
template <> struct MPair<11, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[29]), 1.0, mu[30])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[28]), -1.0, mu[29])); }
};
template <> struct MPair<11, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[3]), -6.0, mu[4])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[33]), -1.0, mu[34])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[32]), 1.0, mu[33])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[31]), -1.0, mu[32])); }
};
template <> struct MPair<11, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[10]), 9.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[50]), -1.0, mu[59]), 1.0, mu[60])); emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[49]), -1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[49]), 1.0, mu[58]), -1.0, mu[59])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[48]), 1.0, mu[49])); }
};
template <> struct MPair<11, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[12]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[53]), -1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[52]), -1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[51]), 1.0, mu[52]), 1.0, mu[65]), -1.0, mu[66])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[51]), 1.0, mu[52])); }
};
template <> struct MPair<11, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][2], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[7]), -9.0, mu[8]), -9.0, mu[13]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54]), -1.0, mu[68]), 1.0, mu[69])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[44]), 1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[3][0], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53]), 1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[43]), -1.0, mu[52]), 1.0, mu[53])); }
};
template <> struct MPair<11, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[10]), -9.0, mu[11]), -9.0, mu[12]), 9.0, mu[13])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[63]), -1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[60]), 1.0, mu[62]), -1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[61]), 1.0, mu[62]), 1.0, mu[65]), -1.0, mu[66])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[59]), -1.0, mu[61]), 1.0, mu[62])); }
};
template <> struct MPair<11, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][4], emg_fma(emg_fma(emg_fma(emg_mul(9.0, mu[10]), -9.0, mu[11]), -9.0, mu[13]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64]), -1.0, mu[68]), 1.0, mu[69])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[60]), 1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[3][1], emg_fma(emg_fma(emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63]), 1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[59]), -1.0, mu[62]), 1.0, mu[63])); }
};
template <> struct MPair<11, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][5], emg_fma(emg_fma(emg_mul(9.0, mu[12]), -18.0, mu[13]), 9.0, mu[14])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_fma(emg_mul(1.0, mu[67]), -2.0, mu[68]), 1.0, mu[69])); emg_mac(acc, G[2][3], emg_fma(emg_fma(emg_mul(-1.0, mu[66]), 2.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][2], emg_fma(emg_fma(emg_mul(-1.0, mu[66]), 2.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[3][3], emg_fma(emg_fma(emg_mul(1.0, mu[65]), -2.0, mu[66]), 1.0, mu[67])); }
};
template <> struct MPair<11, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(-3.0, mu[12]), 3.0, mu[13])); emg_mac(acc, H[5][1], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); emg_mac(acc, H[5][3], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[53])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[51]), 1.0, mu[52])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<11, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[5][2], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<11, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[5][2], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[51]), -1.0, mu[52])); }
};
template <> struct MPair<11, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[5][4], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[61]), -1.0, mu[62])); }
};
template <> struct MPair<11, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[5][1], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); emg_mac(acc, H[5][3], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[63])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[61]), 1.0, mu[62])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<11, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][0], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); emg_mac(acc, H[5][4], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<11, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][1], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[12]), -6.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[51]), -1.0, mu[52])); }
};
template <> struct MPair<11, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[5][3], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[12]), -6.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[61]), -1.0, mu[62])); }
};
template <> struct MPair<12, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][0], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][0], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[20])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[17])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[19])); emg_mac(acc, G[2][1], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<12, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][1], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[22])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[17])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<12, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][2], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[17])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<12, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[22])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<12, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<12, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_mul(-2.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[2])); emg_mac(acc, H[3][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[22])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<12, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[10])); emg_mac(acc, H[1][0], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); emg_mac(acc, H[3][0], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[40])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<12, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[12])); emg_mac(acc, H[1][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); emg_mac(acc, H[3][1], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[42]), -1.0, mu[51])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[42])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<12, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(-3.0, mu[7]), 3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); emg_mac(acc, H[3][2], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[53])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[37]), 1.0, mu[43])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<12, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(-3.0, mu[10]), 3.0, mu[12])); emg_mac(acc, H[1][3], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); emg_mac(acc, H[3][3], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[51])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<12, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(-3.0, mu[10]), 3.0, mu[13])); emg_mac(acc, H[1][4], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); emg_mac(acc, H[3][4], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[53])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[49])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<12, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(-3.0, mu[12]), 3.0, mu[13])); emg_mac(acc, H[1][5], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); emg_mac(acc, H[3][5], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[53])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[51]), 1.0, mu[52])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<12, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[12])); emg_mac(acc, H[0][1], emg_mul(-1.0, mu[10])); emg_mac(acc, H[0][3], emg_mul(-2.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(-1.0, mu[10])); emg_mac(acc, H[1][1], emg_mul(1.0, mu[9])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(-2.0, mu[7])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][3], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[42])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<12, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(-1.0, mu[10])); emg_mac(acc, H[0][4], emg_mul(-2.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(-1.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(1.0, mu[9])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(-2.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][4], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[43])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[41])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<12, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(-1.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(-2.0, mu[7])); emg_mac(acc, H[1][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][1], emg_mul(-2.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[43])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[42])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<12, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][4], emg_mul(-1.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(-2.0, mu[10])); emg_mac(acc, H[1][3], emg_mul(-1.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(1.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[9])); emg_mac(acc, H[3][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[49])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[48])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<12, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[12])); emg_mac(acc, H[0][1], emg_mul(-2.0, mu[10])); emg_mac(acc, H[0][3], emg_mul(-1.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(1.0, mu[10])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[1][3], emg_mul(1.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(2.0, mu[7])); emg_mac(acc, H[3][1], emg_mul(4.0, mu[6])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[48])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<12, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(-2.0, mu[10])); emg_mac(acc, H[0][4], emg_mul(-1.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(1.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[1][4], emg_mul(1.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(2.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(4.0, mu[6])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[49])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[47])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<12, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(-2.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(-1.0, mu[7])); emg_mac(acc, H[1][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(1.0, mu[6])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(4.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[52])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[42])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<12, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][4], emg_mul(-2.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(-1.0, mu[10])); emg_mac(acc, H[1][3], emg_mul(1.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(1.0, mu[9])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[3][4], emg_mul(4.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[52])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[48])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<13, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][0], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[21])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[19])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<13, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][1], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<13, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[24])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<13, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<13, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[24])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<13, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[2])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[24])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<13, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[2][0], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); emg_mac(acc, H[4][0], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<13, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); emg_mac(acc, H[4][1], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<13, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[44])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<13, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[2][3], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); emg_mac(acc, H[4][3], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<13, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<13, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[2][5], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<13, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[0][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-1.0, mu[10])); emg_mac(acc, H[2][1], emg_mul(1.0, mu[9])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(-2.0, mu[7])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][3], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[43])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[40])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<13, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(-1.0, mu[11])); emg_mac(acc, H[0][4], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-1.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(1.0, mu[9])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[44])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<13, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][1], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[44])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<13, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][4], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(-2.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(-1.0, mu[11])); emg_mac(acc, H[2][4], emg_mul(1.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[9])); emg_mac(acc, H[4][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[50])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<13, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[0][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(1.0, mu[10])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[2][3], emg_mul(1.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[7])); emg_mac(acc, H[4][1], emg_mul(4.0, mu[6])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[49])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[46])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<13, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(-2.0, mu[11])); emg_mac(acc, H[0][4], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(1.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[2][4], emg_mul(1.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[6])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[50])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<13, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(-2.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(1.0, mu[6])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[53])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<13, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][4], emg_mul(-2.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(-1.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(1.0, mu[11])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(1.0, mu[9])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[53])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<14, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][0], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[21])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<14, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[23])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[22])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<14, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[24])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[18])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<14, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][3], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[23])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[22])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<14, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[24])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<14, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_mul(-2.0, mu[4])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[24])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[22])); }
};
template <> struct MPair<14, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[2][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[5][0], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[41]), -1.0, mu[47])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[41])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[40])); }
};
template <> struct MPair<14, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[5][1], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[43]), -1.0, mu[52])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[43])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[42]), 1.0, mu[51])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[42])); }
};
template <> struct MPair<14, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[5]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[44]), -1.0, mu[54])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[38]), 1.0, mu[44])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[43])); }
};
template <> struct MPair<14, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[2][3], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[5][3], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[52])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[49])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[51])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48])); }
};
template <> struct MPair<14, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[54])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[49])); }
};
template <> struct MPair<14, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[2][5], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[54])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[51]), -1.0, mu[52])); }
};
template <> struct MPair<14, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[1][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[1][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-1.0, mu[12])); emg_mac(acc, H[2][1], emg_mul(1.0, mu[10])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[5][3], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[43])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[42])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<14, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(-1.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-2.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[44])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<14, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(-1.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(-2.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(-1.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(1.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(-2.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[44])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[42])); }
};
template <> struct MPair<14, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][4], emg_mul(-1.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(-2.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(-1.0, mu[13])); emg_mac(acc, H[2][4], emg_mul(1.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[50])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<14, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[1][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[1][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(1.0, mu[12])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][3], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(4.0, mu[6])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[49])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[48])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<14, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(-2.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[6])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[50])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<14, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(-2.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(-1.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(1.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[53])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[42])); }
};
template <> struct MPair<14, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][4], emg_mul(-2.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(-1.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(1.0, mu[13])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(1.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[53])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<15, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][0], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[27])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[26])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<15, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[28])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<15, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[30])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<15, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][3], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[29])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[28])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<15, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[30])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<15, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_mul(-2.0, mu[4])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[30])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[28])); }
};
template <> struct MPair<15, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[11])); emg_mac(acc, H[4][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[5][0], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[57])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[47])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[56])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); }
};
template <> struct MPair<15, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[13])); emg_mac(acc, H[4][1], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[5][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[62])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[49])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[61])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[48])); }
};
template <> struct MPair<15, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_fma(emg_mul(-3.0, mu[8]), 3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[5][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[64])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[49])); }
};
template <> struct MPair<15, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[13])); emg_mac(acc, H[4][3], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[5][3], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[58]), 1.0, mu[61])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[58])); }
};
template <> struct MPair<15, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_fma(emg_mul(-3.0, mu[11]), 3.0, mu[14])); emg_mac(acc, H[4][4], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[5][4], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[59])); }
};
template <> struct MPair<15, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_fma(emg_mul(-3.0, mu[13]), 3.0, mu[14])); emg_mac(acc, H[4][5], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[2][3], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[61]), -1.0, mu[62])); }
};
template <> struct MPair<15, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[3][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[3][3], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(-1.0, mu[12])); emg_mac(acc, H[4][1], emg_mul(1.0, mu[10])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-2.0, mu[10])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[5][3], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[49])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[48])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<15, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(-1.0, mu[11])); emg_mac(acc, H[3][4], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-2.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[50])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<15, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(-1.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(-2.0, mu[8])); emg_mac(acc, H[4][1], emg_mul(-1.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(1.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[50])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<15, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][4], emg_mul(-1.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(-2.0, mu[11])); emg_mac(acc, H[4][3], emg_mul(-1.0, mu[13])); emg_mac(acc, H[4][4], emg_mul(1.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(-2.0, mu[11])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(4.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][2], emg_mul(1.0, mu[60])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[58])); }
};
template <> struct MPair<15, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[3][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[3][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(1.0, mu[12])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[10])); emg_mac(acc, H[4][3], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][1], emg_mul(4.0, mu[9])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[59])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[58])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<15, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(-2.0, mu[11])); emg_mac(acc, H[3][4], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[4][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[9])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[60])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<15, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(-2.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][1], emg_mul(1.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(4.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][0], emg_mul(1.0, mu[63])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<15, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][4], emg_mul(-2.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(-1.0, mu[11])); emg_mac(acc, H[4][3], emg_mul(1.0, mu[13])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(1.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[11])); emg_mac(acc, H[5][4], emg_mul(4.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[2][1], emg_mul(1.0, mu[63])); emg_mac(acc, G[2][3], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[58])); }
};
template <> struct MPair<16, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][0], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][0], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[26])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[19])); emg_mac(acc, G[2][1], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<16, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[28])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<16, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<16, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][3], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[28])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[26])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<16, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][4], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[26])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<16, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_mul(2.0, mu[3])); emg_mac(acc, H[1][5], emg_mul(4.0, mu[2])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[28])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<16, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[10])); emg_mac(acc, H[1][0], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); emg_mac(acc, H[3][0], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[56])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[2][1], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<16, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[12])); emg_mac(acc, H[1][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); emg_mac(acc, H[3][1], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[61])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<16, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[13])); emg_mac(acc, H[1][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); emg_mac(acc, H[3][2], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[63])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[49])); emg_mac(acc, G[2][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<16, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[12])); emg_mac(acc, H[1][3], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); emg_mac(acc, H[3][3], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[58]), -1.0, mu[61])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[58])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[2][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<16, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[13])); emg_mac(acc, H[1][4], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); emg_mac(acc, H[3][4], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[63])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[56]), 1.0, mu[59])); emg_mac(acc, G[2][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<16, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(3.0, mu[12]), -3.0, mu[13])); emg_mac(acc, H[1][5], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); emg_mac(acc, H[3][5], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[63])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[61]), 1.0, mu[62])); emg_mac(acc, G[2][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[2][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<16, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[12])); emg_mac(acc, H[0][1], emg_mul(1.0, mu[10])); emg_mac(acc, H[0][3], emg_mul(2.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(-2.0, mu[10])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[1][3], emg_mul(4.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(-1.0, mu[7])); emg_mac(acc, H[3][1], emg_mul(1.0, mu[6])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[48])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[40])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<16, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(-2.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[1][4], emg_mul(4.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(-1.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(1.0, mu[6])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[49])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[41])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<16, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(1.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[7])); emg_mac(acc, H[1][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(4.0, mu[6])); emg_mac(acc, H[3][1], emg_mul(-1.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(1.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[49])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[48])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<16, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][4], emg_mul(1.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][3], emg_mul(-2.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(4.0, mu[9])); emg_mac(acc, H[3][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[3][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[59])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[58])); emg_mac(acc, G[2][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<16, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[12])); emg_mac(acc, H[0][1], emg_mul(2.0, mu[10])); emg_mac(acc, H[0][3], emg_mul(1.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(2.0, mu[10])); emg_mac(acc, H[1][1], emg_mul(4.0, mu[9])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(1.0, mu[7])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][3], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[58])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<16, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[0][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[1][0], emg_mul(2.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(4.0, mu[9])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][0], emg_mul(1.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][4], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[59])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[46])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[47])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<16, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(1.0, mu[7])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[1][2], emg_mul(4.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[6])); emg_mac(acc, H[3][1], emg_mul(1.0, mu[8])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[62])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[48])); emg_mac(acc, G[2][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<16, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[12])); emg_mac(acc, H[0][5], emg_mul(1.0, mu[10])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(4.0, mu[10])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[9])); emg_mac(acc, H[3][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[3][5], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[62])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[58])); emg_mac(acc, G[2][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[2][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<17, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][0], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[27])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[19])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<17, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][1], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<17, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[30])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[16])); }
};
template <> struct MPair<17, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][3], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<17, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[30])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[27])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[19])); }
};
template <> struct MPair<17, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[2])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[30])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[21])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<17, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[2][0], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[9])); emg_mac(acc, H[4][0], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[47]), -1.0, mu[57])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[47])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[39]), 1.0, mu[45])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[39])); }
};
template <> struct MPair<17, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[10])); emg_mac(acc, H[4][1], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[62])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[49])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[48])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[40])); }
};
template <> struct MPair<17, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][2], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[6]), -6.0, mu[11])); emg_mac(acc, H[4][2], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[50]), -1.0, mu[64])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[41]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[36]), -1.0, mu[41])); }
};
template <> struct MPair<17, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[2][3], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[10])); emg_mac(acc, H[4][3], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[59]), -1.0, mu[62])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[59])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[48])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[46])); }
};
template <> struct MPair<17, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][4], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[9]), -6.0, mu[11])); emg_mac(acc, H[4][4], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[60]), -1.0, mu[64])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[57]), 1.0, mu[60])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[47]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[45]), -1.0, mu[47])); }
};
template <> struct MPair<17, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][5], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[11])); emg_mac(acc, H[4][5], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[64])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[50])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[48]), -1.0, mu[49])); }
};
template <> struct MPair<17, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[0][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[0][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-2.0, mu[10])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[2][3], emg_mul(4.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(-1.0, mu[7])); emg_mac(acc, H[4][1], emg_mul(1.0, mu[6])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[49])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[40])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<17, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(1.0, mu[11])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-2.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(1.0, mu[6])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[50])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<17, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(-2.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[6])); emg_mac(acc, H[4][1], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(1.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[50])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[41])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<17, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[0][4], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(2.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(-2.0, mu[11])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[9])); emg_mac(acc, H[4][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[4][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[60])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<17, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[0][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[0][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][1], emg_mul(4.0, mu[9])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(1.0, mu[7])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][3], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[59])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[46])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<17, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[11])); emg_mac(acc, H[0][4], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[9])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][0], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][4], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[60])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[47])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[39])); }
};
template <> struct MPair<17, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][2], emg_mul(2.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[6])); emg_mac(acc, H[4][1], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[63])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<17, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[0][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[0][4], emg_mul(2.0, mu[13])); emg_mac(acc, H[0][5], emg_mul(1.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[11])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[10])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[9])); emg_mac(acc, H[4][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[4][5], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[63])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<18, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][0], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[0][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[20])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<18, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][1], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[32])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[22])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<18, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[33])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[17])); }
};
template <> struct MPair<18, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][3], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[32])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[22])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<18, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[33])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<18, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_mul(2.0, mu[4])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[1])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[33])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[32])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[22])); }
};
template <> struct MPair<18, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[2][0], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[10])); emg_mac(acc, H[5][0], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[59])); emg_mac(acc, G[0][1], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[49])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[40]), 1.0, mu[46])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[40])); }
};
template <> struct MPair<18, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[2][1], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[12])); emg_mac(acc, H[5][1], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[66])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[52])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[42]), 1.0, mu[51])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[42])); }
};
template <> struct MPair<18, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][2], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[2][2], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[13])); emg_mac(acc, H[5][2], emg_fma(emg_mul(3.0, mu[5]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[68])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[37]), -1.0, mu[43])); }
};
template <> struct MPair<18, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[2][3], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[12])); emg_mac(acc, H[5][3], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[7])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[66])); emg_mac(acc, G[0][2], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[62])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[51])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[48])); }
};
template <> struct MPair<18, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][4], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[2][4], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[13])); emg_mac(acc, H[5][4], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[68])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[46]), -1.0, mu[49])); }
};
template <> struct MPair<18, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][5], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[2][5], emg_fma(emg_mul(6.0, mu[12]), -6.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(3.0, mu[7]), -3.0, mu[8])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_fma(emg_mul(1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[0][3], emg_fma(emg_mul(-1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[52]), 1.0, mu[53])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[51]), -1.0, mu[52])); }
};
template <> struct MPair<18, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[1][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[1][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-2.0, mu[12])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][3], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-1.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(1.0, mu[6])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[52])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[42])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<18, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(1.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(-2.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-1.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(1.0, mu[6])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[53])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<18, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(1.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(-2.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(2.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(-1.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[53])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[43])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[42])); }
};
template <> struct MPair<18, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[1][4], emg_mul(1.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(2.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(-2.0, mu[13])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(4.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(-1.0, mu[8])); emg_mac(acc, H[5][4], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][2], emg_mul(1.0, mu[63])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<18, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[1][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[1][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[12])); emg_mac(acc, H[2][1], emg_mul(4.0, mu[10])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(1.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[6])); emg_mac(acc, H[5][3], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[62])); emg_mac(acc, G[0][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[48])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<18, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[11])); emg_mac(acc, H[1][4], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][0], emg_mul(2.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[10])); emg_mac(acc, H[2][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(1.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[6])); emg_mac(acc, H[5][4], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[63])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[40])); }
};
template <> struct MPair<18, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][2], emg_mul(2.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(1.0, mu[8])); emg_mac(acc, H[2][1], emg_mul(2.0, mu[13])); emg_mac(acc, H[2][2], emg_mul(4.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(1.0, mu[8])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(1.0, mu[5])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][0], emg_mul(1.0, mu[67])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[42])); }
};
template <> struct MPair<18, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[1][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[1][4], emg_mul(2.0, mu[13])); emg_mac(acc, H[1][5], emg_mul(1.0, mu[11])); emg_mac(acc, H[2][3], emg_mul(2.0, mu[13])); emg_mac(acc, H[2][4], emg_mul(4.0, mu[12])); emg_mac(acc, H[2][5], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][5], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[0][1], emg_mul(1.0, mu[67])); emg_mac(acc, G[0][3], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<19, 0> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][0], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][0], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[29])); emg_mac(acc, G[1][1], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[26])); emg_mac(acc, G[3][1], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<19, 1> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][1], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[32])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[28])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<19, 2> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[33])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[23])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[20])); }
};
template <> struct MPair<19, 3> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][3], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[32])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[28])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<19, 4> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[33])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[26])); }
};
template <> struct MPair<19, 5> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_mul(2.0, mu[4])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[3])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[2])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[33])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[32])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[29])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[28])); }
};
template <> struct MPair<19, 6> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[11])); emg_mac(acc, H[4][0], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[10])); emg_mac(acc, H[5][0], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[49]), -1.0, mu[59])); emg_mac(acc, G[1][1], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[49])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[46]), 1.0, mu[56])); emg_mac(acc, G[3][1], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[46])); }
};
template <> struct MPair<19, 7> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[13])); emg_mac(acc, H[4][1], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[12])); emg_mac(acc, H[5][1], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[52]), -1.0, mu[66])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[52])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[48]), 1.0, mu[61])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[48])); }
};
template <> struct MPair<19, 8> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][2], emg_fma(emg_mul(3.0, mu[8]), -3.0, mu[14])); emg_mac(acc, H[4][2], emg_fma(emg_mul(6.0, mu[7]), -6.0, mu[13])); emg_mac(acc, H[5][2], emg_fma(emg_mul(3.0, mu[6]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_fma(emg_mul(1.0, mu[53]), -1.0, mu[68])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[43]), 1.0, mu[53])); emg_mac(acc, G[3][0], emg_fma(emg_mul(-1.0, mu[49]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[40]), -1.0, mu[49])); }
};
template <> struct MPair<19, 9> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[13])); emg_mac(acc, H[4][3], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[12])); emg_mac(acc, H[5][3], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[10])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[62]), -1.0, mu[66])); emg_mac(acc, G[1][2], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[62])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[58]), 1.0, mu[61])); emg_mac(acc, G[3][2], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[58])); }
};
template <> struct MPair<19, 10> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][4], emg_fma(emg_mul(3.0, mu[11]), -3.0, mu[14])); emg_mac(acc, H[4][4], emg_fma(emg_mul(6.0, mu[10]), -6.0, mu[13])); emg_mac(acc, H[5][4], emg_fma(emg_mul(3.0, mu[9]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_fma(emg_mul(1.0, mu[63]), -1.0, mu[68])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][1], emg_fma(emg_mul(-1.0, mu[59]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[56]), -1.0, mu[59])); }
};
template <> struct MPair<19, 11> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][5], emg_fma(emg_mul(3.0, mu[13]), -3.0, mu[14])); emg_mac(acc, H[4][5], emg_fma(emg_mul(6.0, mu[12]), -6.0, mu[13])); emg_mac(acc, H[5][5], emg_fma(emg_mul(3.0, mu[10]), -3.0, mu[11])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_fma(emg_mul(1.0, mu[67]), -1.0, mu[68])); emg_mac(acc, G[1][3], emg_fma(emg_mul(-1.0, mu[66]), 1.0, mu[67])); emg_mac(acc, G[3][2], emg_fma(emg_mul(-1.0, mu[62]), 1.0, mu[63])); emg_mac(acc, G[3][3], emg_fma(emg_mul(1.0, mu[61]), -1.0, mu[62])); }
};
template <> struct MPair<19, 12> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-1.0, mu[13])); emg_mac(acc, H[3][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[3][3], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(-2.0, mu[12])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[10])); emg_mac(acc, H[4][3], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-1.0, mu[10])); emg_mac(acc, H[5][1], emg_mul(1.0, mu[9])); emg_mac(acc, H[5][3], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[52])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[48])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<19, 13> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(1.0, mu[11])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(-2.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(-1.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(1.0, mu[9])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[53])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<19, 14> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(1.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[8])); emg_mac(acc, H[4][1], emg_mul(-2.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(2.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(-1.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(1.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[53])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<19, 15> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(-1.0, mu[14])); emg_mac(acc, H[3][4], emg_mul(1.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(2.0, mu[11])); emg_mac(acc, H[4][3], emg_mul(-2.0, mu[13])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(4.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(-1.0, mu[11])); emg_mac(acc, H[5][4], emg_mul(1.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(2.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][2], emg_mul(1.0, mu[63])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][2], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[58])); }
};
template <> struct MPair<19, 16> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(1.0, mu[13])); emg_mac(acc, H[3][1], emg_mul(2.0, mu[11])); emg_mac(acc, H[3][3], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[12])); emg_mac(acc, H[4][1], emg_mul(4.0, mu[10])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(1.0, mu[10])); emg_mac(acc, H[5][1], emg_mul(2.0, mu[9])); emg_mac(acc, H[5][3], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[62])); emg_mac(acc, G[1][2], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[58])); emg_mac(acc, G[3][2], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<19, 17> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][0], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[11])); emg_mac(acc, H[3][4], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][0], emg_mul(2.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[10])); emg_mac(acc, H[4][4], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][0], emg_mul(1.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[9])); emg_mac(acc, H[5][4], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[63])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[49])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[59])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[46])); }
};
template <> struct MPair<19, 18> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][1], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][2], emg_mul(2.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(1.0, mu[8])); emg_mac(acc, H[4][1], emg_mul(2.0, mu[13])); emg_mac(acc, H[4][2], emg_mul(4.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[7])); emg_mac(acc, H[5][1], emg_mul(1.0, mu[11])); emg_mac(acc, H[5][2], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(1.0, mu[6])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][0], emg_mul(1.0, mu[67])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[52])); emg_mac(acc, G[3][0], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[48])); }
};
template <> struct MPair<19, 19> {
  template <class A, class T, class R> __device__ __forceinline__ static void stiff(A &acc, const T &H, const R *mu) { emg_mac(acc, H[3][3], emg_mul(1.0, mu[14])); emg_mac(acc, H[3][4], emg_mul(2.0, mu[13])); emg_mac(acc, H[3][5], emg_mul(1.0, mu[11])); emg_mac(acc, H[4][3], emg_mul(2.0, mu[13])); emg_mac(acc, H[4][4], emg_mul(4.0, mu[12])); emg_mac(acc, H[4][5], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][3], emg_mul(1.0, mu[11])); emg_mac(acc, H[5][4], emg_mul(2.0, mu[10])); emg_mac(acc, H[5][5], emg_mul(1.0, mu[9])); }
  template <class A, class T, class R> __device__ __forceinline__ static void mass(A &acc, const T &G, const R *mu) { emg_mac(acc, G[1][1], emg_mul(1.0, mu[67])); emg_mac(acc, G[1][3], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][1], emg_mul(-1.0, mu[62])); emg_mac(acc, G[3][3], emg_mul(1.0, mu[58])); }
};
}  // namespace emg_mtables
