// Small fixed-radix DFTs on registers (radix 2, 3, 4, 5), shared by the
// shared-memory line FFTs and the warp-level FFTs.
// Sign: forward e^{-2 pi i / r}, inverse e^{+2 pi i / r}; unnormalised.
#pragma once

#include "fvr_common.cuh"

namespace fvr {

template <typename T>
__device__ __forceinline__ Cx<T> mul_i(Cx<T> a, bool neg) {  // +i*a  or  -i*a
  return neg ? Cx<T>{a.y, -a.x} : Cx<T>{-a.y, a.x};
}

template <typename T, int R>
struct Dft;

template <typename T>
struct Dft<T, 2> {
  __device__ __forceinline__ static void run(Cx<T> (&v)[2], bool) {
    Cx<T> a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};

template <typename T>
struct Dft<T, 4> {
  __device__ __forceinline__ static void run(Cx<T> (&v)[4], bool inv) {
    Cx<T> a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    Cx<T> c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    Cx<T> id = mul_i(d, !inv);  // forward: -i d
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, id);
    v[3] = csub(b, id);
  }
};

template <typename T>
struct Dft<T, 3> {
  __device__ __forceinline__ static void run(Cx<T> (&v)[3], bool inv) {
    const T s3 = static_cast<T>(0.86602540378443864676372317075294);  // sqrt(3)/2
    Cx<T> t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    Cx<T> m{v[0].x - static_cast<T>(0.5) * t1.x, v[0].y - static_cast<T>(0.5) * t1.y};
    Cx<T> st{s3 * t2.x, s3 * t2.y};
    Cx<T> ist = mul_i(st, !inv);  // forward: -i s t2
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, ist);
    v[2] = csub(m, ist);
  }
};

template <typename T>
struct Dft<T, 5> {
  __device__ __forceinline__ static void run(Cx<T> (&v)[5], bool inv) {
    const T c1 = static_cast<T>(0.30901699437494742410229341718282);   // cos(2pi/5)
    const T c2 = static_cast<T>(-0.80901699437494742410229341718282);  // cos(4pi/5)
    const T s1 = static_cast<T>(0.95105651629515357211643933337938);   // sin(2pi/5)
    const T s2 = static_cast<T>(0.58778525229247312916870595463907);   // sin(4pi/5)
    Cx<T> t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    Cx<T> t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    Cx<T> a1{v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y};
    Cx<T> a2{v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y};
    Cx<T> b1{s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y};
    Cx<T> b2{s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y};
    Cx<T> ib1 = mul_i(b1, !inv), ib2 = mul_i(b2, !inv);  // forward: -i b
    v[0] = Cx<T>{v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y};
    v[1] = cadd(a1, ib1);
    v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[3] = csub(a2, ib2);
  }
};

}  // namespace fvr
