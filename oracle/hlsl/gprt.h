// gprt.h -- TEST INFRASTRUCTURE ONLY: a host stand-in for the GPRT device API, so that the
// reference's own HLSL programs (deviceCodeRBF/Splat/Common/Bounds.hlsl with sharedCode.h and
// rng.h) compile as C++ and run on the CPU. The reference's GPRT submodule is not vendored; this
// header is written from the HLSL language and from how the reference's programs use GPRT.
//
// It is included textually inside a namespace (one per reference module, see href_*.cpp), after
// the translation unit has included every standard header it needs, so it includes none itself.
//
// What the GPU runtime would decide is fixed here by the same documented model the oracle and the
// CUDA path use (so a comparison pins the oracle's restatement of the reference's control flow and
// arithmetic, not a choice of vendor math):
//  - exp / log / pow: the oracle's orc_expf / orc_logf / orc_powf, with pow(x, 2) = x x and
//    pow(x, 3) = (x x) x (a compiler's strength reduction of small integer exponents);
//  - sqrt-based length / distance / normalize: v / sqrt((x x + y y) + z z);
//  - sin / cos: the C library's sinf / cosf; ldexp: ldexpf;
//  - min / max: fminf / fmaxf; lerp(x, y, s) = x + s (y - x);
//  - Texture1D::SampleGrad: the oracle's orc_tex_sample (linear between texel centres, clamp to
//    edge) on the decoded texel values; Texture2D::SampleGrad: bilinear with clamp to edge and
//    weights rounded to multiples of 1/256 (the sub-texel precision of texture units), so a
//    coordinate at a texel centre returns that texel exactly;
//  - make_bgra: saturate, round half up to 8 bits, B | G << 8 | R << 16 | A << 24;
//  - TraceRay: brute force over the leaf boxes of the bounds program in leaf order (or reverse
//    leaf order, to expose results that depend on the hardware's traversal order); a zero-length
//    ray visits the boxes containing its origin, a ray segment the boxes it overlaps; ReportHit
//    calls the any-hit program for hits within [RayTMin, RayTCurrent], a hit the any-hit program
//    does not ignore becomes the closest hit (RayTCurrent = t), acceptHitAndEndSearch ends the
//    traversal.

typedef unsigned int uint;

extern "C" float orc_expf(float x);
extern "C" float orc_logf(float x);
extern "C" float orc_powf(float x, float y);
extern "C" float orc_tex_sample(const float *tex, int n, int stride, int channel, float u);

// ---- vector types ------------------------------------------------------------------------------

struct float2;
struct float3;
struct float4;
struct int2;
struct uint2;
struct uint3;

struct bool2 {
  bool x, y;
};
struct bool3 {
  bool x, y, z;
};
inline bool all(bool2 b) { return b.x && b.y; }
inline bool all(bool3 b) { return b.x && b.y && b.z; }
inline bool any(bool2 b) { return b.x || b.y; }
inline bool any(bool3 b) { return b.x || b.y || b.z; }

// swizzle proxies: storage that aliases leading components of the enclosing vector
template <class V, class S, int N>
struct Lead {
  S v[N];
  operator V() const;
  Lead &operator=(const V &o);
  Lead &operator+=(const V &o);
};

struct float2 {
  union {
    struct { float x, y; };
    struct { float r, g; };
  };
  float2() : x(0), y(0) {}
  template <class A, class B>
  float2(A a, B b) : x((float)a), y((float)b) {}
  float2(const int2 &o);
  float2(const uint2 &o);
  float2(const Lead<int2, int, 2> &o);
  float &operator[](int i) { return i == 0 ? x : y; }
  float operator[](int i) const { return i == 0 ? x : y; }
};

struct float3 {
  union {
    struct { float x, y, z; };
    struct { float r, g, b; };
    Lead<float2, float, 2> xy;
  };
  float3() : x(0), y(0), z(0) {}
  template <class A, class B, class C>
  float3(A a, B b, C c) : x((float)a), y((float)b), z((float)c) {}
  explicit float3(const uint3 &o);
  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

struct float4 {
  union {
    struct { float x, y, z, w; };
    struct { float r, g, b, a; };
    Lead<float3, float, 3> xyz;
    Lead<float3, float, 3> rgb;
    Lead<float2, float, 2> xy;
  };
  float4() : x(0), y(0), z(0), w(0) {}
  template <class A, class B, class C, class D>
  float4(A a, B b, C c, D d) : x((float)a), y((float)b), z((float)c), w((float)d) {}
  float4(const float3 &v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

struct int2 {
  union {
    struct { int x, y; };
    Lead<int2, int, 2> xy;
  };
  int2() : x(0), y(0) {}
  template <class A, class B>
  int2(A a, B b) : x((int)a), y((int)b) {}
  int2(const uint2 &o);
  int2(const Lead<uint2, uint, 2> &o);
  int2(const int2 &o) : x(o.x), y(o.y) {}
  int2 &operator=(const int2 &o) {
    x = o.x;
    y = o.y;
    return *this;
  }
};

struct uint2 {
  union {
    struct { uint x, y; };
    Lead<uint2, uint, 2> xy;
  };
  uint2() : x(0), y(0) {}
  template <class A, class B>
  uint2(A a, B b) : x((uint)a), y((uint)b) {}
  uint2(const int2 &o) : x((uint)o.x), y((uint)o.y) {}
  uint2(const uint2 &o) : x(o.x), y(o.y) {}
  uint2 &operator=(const uint2 &o) {
    x = o.x;
    y = o.y;
    return *this;
  }
};

struct uint3 {
  union {
    struct { uint x, y, z; };
    Lead<uint2, uint, 2> xy;
  };
  uint3() : x(0), y(0), z(0) {}
  template <class A, class B, class C>
  uint3(A a, B b, C c) : x((uint)a), y((uint)b), z((uint)c) {}
};

template <class V, class S, int N>
inline Lead<V, S, N>::operator V() const {
  V o;
  S *d = reinterpret_cast<S *>(&o);
  for (int i = 0; i < N; ++i) d[i] = v[i];
  return o;
}
template <class V, class S, int N>
inline Lead<V, S, N> &Lead<V, S, N>::operator=(const V &o) {
  const S *s = reinterpret_cast<const S *>(&o);
  for (int i = 0; i < N; ++i) v[i] = s[i];
  return *this;
}
template <class V, class S, int N>
inline Lead<V, S, N> &Lead<V, S, N>::operator+=(const V &o) {
  const S *s = reinterpret_cast<const S *>(&o);
  for (int i = 0; i < N; ++i) v[i] = v[i] + s[i];
  return *this;
}

inline float2::float2(const int2 &o) : x((float)o.x), y((float)o.y) {}
inline float2::float2(const uint2 &o) : x((float)o.x), y((float)o.y) {}
inline float2::float2(const Lead<int2, int, 2> &o) : x((float)o.v[0]), y((float)o.v[1]) {}
inline float3::float3(const uint3 &o) : x((float)o.x), y((float)o.y), z((float)o.z) {}
inline int2::int2(const uint2 &o) : x((int)o.x), y((int)o.y) {}
inline int2::int2(const Lead<uint2, uint, 2> &o) : x((int)o.v[0]), y((int)o.v[1]) {}

// the vector types, their scalar type and size
template <class V>
struct href_vec {
  static const bool value = false;
};
#define HREF_VEC(V, T, N)       \
  template <>                   \
  struct href_vec<V> {          \
    static const bool value = true; \
    typedef T scalar;           \
    static const int n = N;     \
  };
HREF_VEC(float2, float, 2)
HREF_VEC(float3, float, 3)
HREF_VEC(float4, float, 4)
HREF_VEC(int2, int, 2)
HREF_VEC(uint2, uint, 2)
#undef HREF_VEC

template <class V, class S>
using vec_scalar = typename std::enable_if<href_vec<V>::value && std::is_arithmetic<S>::value, V>::type;
template <class S>
using arith = typename std::enable_if<std::is_arithmetic<S>::value, int>::type;

template <class V, class F>
inline V href_map2(const V &a, const V &b, F f) {
  typedef typename href_vec<V>::scalar T;
  V o;
  for (int i = 0; i < href_vec<V>::n; ++i)
    reinterpret_cast<T *>(&o)[i] = f(reinterpret_cast<const T *>(&a)[i], reinterpret_cast<const T *>(&b)[i]);
  return o;
}

// vector op vector: one non-template function per type, so an int2 meets a float2 as float2 and
// a swizzle meets its vector type through its conversion
#define HREF_VV(V)                                                                                          \
  inline V operator+(const V &a, const V &b) { return href_map2(a, b, [](auto x, auto y) { return x + y; }); } \
  inline V operator-(const V &a, const V &b) { return href_map2(a, b, [](auto x, auto y) { return x - y; }); } \
  inline V operator*(const V &a, const V &b) { return href_map2(a, b, [](auto x, auto y) { return x * y; }); } \
  inline V operator/(const V &a, const V &b) { return href_map2(a, b, [](auto x, auto y) { return x / y; }); } \
  inline V operator-(const V &a) { return href_map2(a, a, [](auto x, auto) { return -x; }); }              \
  inline V &operator+=(V &a, const V &b) { return a = a + b; }                                              \
  inline V &operator-=(V &a, const V &b) { return a = a - b; }                                              \
  inline V &operator*=(V &a, const V &b) { return a = a * b; }                                              \
  inline V &operator/=(V &a, const V &b) { return a = a / b; }
HREF_VV(float2)
HREF_VV(float3)
HREF_VV(float4)
HREF_VV(int2)
HREF_VV(uint2)
#undef HREF_VV

// vector op scalar: templates on the exact vector type (the scalar converts to the vector's type)
template <class V, class S>
inline vec_scalar<V, S> href_vs(const V &a, S s, int op) {
  typedef typename href_vec<V>::scalar T;
  const T t = (T)s;
  return href_map2(a, a, [t, op](T x, T) { return op == 0 ? x + t : op == 1 ? x - t : op == 2 ? x * t : x / t; });
}
template <class V, class S>
inline vec_scalar<V, S> operator+(const V &a, S s) { return href_vs(a, s, 0); }
template <class V, class S>
inline vec_scalar<V, S> operator-(const V &a, S s) { return href_vs(a, s, 1); }
template <class V, class S>
inline vec_scalar<V, S> operator*(const V &a, S s) { return href_vs(a, s, 2); }
template <class V, class S>
inline vec_scalar<V, S> operator/(const V &a, S s) { return href_vs(a, s, 3); }
template <class V, class S>
inline vec_scalar<V, S> operator*(S s, const V &a) {
  typedef typename href_vec<V>::scalar T;
  const T t = (T)s;
  return href_map2(a, a, [t](T x, T) { return t * x; });
}
template <class V, class S>
inline typename std::enable_if<href_vec<V>::value && std::is_arithmetic<S>::value, V &>::type operator*=(V &a, S s) {
  return a = a * s;
}
template <class V, class S>
inline typename std::enable_if<href_vec<V>::value && std::is_arithmetic<S>::value, V &>::type operator/=(V &a, S s) {
  return a = a / s;
}
// swizzle op scalar
template <class V, class E, int N, class S, arith<S> = 0>
inline V operator+(const Lead<V, E, N> &a, S s) { return V(a) + s; }
template <class V, class E, int N, class S, arith<S> = 0>
inline V operator-(const Lead<V, E, N> &a, S s) { return V(a) - s; }
template <class V, class E, int N, class S, arith<S> = 0>
inline V operator*(const Lead<V, E, N> &a, S s) { return V(a) * s; }
template <class V, class E, int N, class S, arith<S> = 0>
inline V operator/(const Lead<V, E, N> &a, S s) { return V(a) / s; }
template <class V, class E, int N, class S, arith<S> = 0>
inline V operator*(S s, const Lead<V, E, N> &a) { return s * V(a); }

inline bool2 operator==(const uint2 &a, const uint2 &b) { return bool2{a.x == b.x, a.y == b.y}; }
inline bool3 operator<=(const float3 &a, const float3 &b) { return bool3{a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bool3 operator>(const float3 &a, const float3 &b) { return bool3{a.x > b.x, a.y > b.y, a.z > b.z}; }

// ---- intrinsics ----------------------------------------------------------------------------------

inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline float3 min(const float3 &a, const float3 &b) { return float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
inline float3 max(const float3 &a, const float3 &b) { return float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
inline float abs(float a) { return fabsf(a); }
inline float3 abs(const float3 &a) { return float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
inline float sign1(float a) { return a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f); }
inline float3 sign(const float3 &a) { return float3(sign1(a.x), sign1(a.y), sign1(a.z)); }
inline float sqrt(float a) { return sqrtf(a); }
inline float exp(float a) { return orc_expf(a); }
inline float log(float a) { return orc_logf(a); }
inline float pow(float x, float y) {
  if (y == 2.0f) return x * x;
  if (y == 3.0f) return (x * x) * x;
  return orc_powf(x, y);
}
inline float3 pow(const float3 &x, float y) { return float3(pow(x.x, y), pow(x.y, y), pow(x.z, y)); }
inline float sin(float a) { return sinf(a); }
inline float cos(float a) { return cosf(a); }
inline float ldexp(float a, int e) { return ldexpf(a, e); }
inline float dot(const float3 &a, const float3 &b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float length(const float3 &a) { return sqrtf(dot(a, a)); }
inline float distance(const float3 &a, const float3 &b) { return length(a - b); }
inline float3 normalize(const float3 &a) {
  float l = length(a);
  return float3(a.x / l, a.y / l, a.z / l);
}
inline float4 lerp(const float4 &x, const float4 &y, float s) { return x + s * (y - x); }
inline float saturate(float v) { return (v > 0.0f) ? (v > 1.0f ? 1.0f : v) : 0.0f; }

// ---- ray tracing state -----------------------------------------------------------------------------

#define RAY_FLAG_NONE 0u

struct RayDesc {
  float3 Origin;
  float TMin;
  float3 Direction;
  float TMax;
};

// one CPU thread runs one program invocation at a time
struct HrefThread {
  uint3 launch_index, launch_dims, dispatch_thread;
  float3 origin, direction;
  float tmin, tcur;
  uint primitive;
  void *payload;
  bool ignored, end_search;
};
inline HrefThread &href_thread() {
  static thread_local HrefThread t;
  return t;
}
inline uint3 DispatchRaysIndex() { return href_thread().launch_index; }
inline uint3 DispatchRaysDimensions() { return href_thread().launch_dims; }
inline float3 WorldRayOrigin() { return href_thread().origin; }
inline float3 WorldRayDirection() { return href_thread().direction; }
inline float RayTMin() { return href_thread().tmin; }
inline float RayTCurrent() { return href_thread().tcur; }
inline uint PrimitiveIndex() { return href_thread().primitive; }
#define DispatchThreadID (href_thread().dispatch_thread)

// The module defines these two after its programs (href_*.cpp): the intersection program of a
// ray type, and the any-hit program called with the payload and a hit attribute.
void href_intersection(int ray_type);
void href_any_hit(void *payload, const void *attribute);

template <class A>
inline bool ReportHit(float t, uint kind, A attribute) {
  (void)kind;
  HrefThread &th = href_thread();
  if (th.end_search || t < th.tmin || t > th.tcur) return false;
  th.ignored = false;
  href_any_hit(th.payload, &attribute);
  if (!th.ignored) th.tcur = t;
  return !th.ignored;
}

// the leaf boxes TraceRay visits (6 floats per leaf: lo xyz, hi xyz; NaN = inactive)
struct HrefScene {
  const float *boxes;
  uint nleaves;
  bool reverse;
};
inline HrefScene &href_scene() {
  static HrefScene s;
  return s;
}

struct RaytracingAccelerationStructure {
  int unused;
};
struct SamplerState {
  int unused;
};

template <class P>
inline void TraceRay(RaytracingAccelerationStructure, uint flags, uint mask, uint ray_type, uint ntypes,
                     uint miss, RayDesc ray, P &payload) {
  (void)flags, (void)mask, (void)ntypes, (void)miss;
  HrefThread &th = href_thread();
  const HrefThread saved = th;
  th.origin = ray.Origin;
  th.direction = ray.Direction;
  th.tmin = ray.TMin;
  th.tcur = ray.TMax;
  th.payload = &payload;
  th.end_search = false;
  const HrefScene &sc = href_scene();
  const float inv[3] = {1.0f / ray.Direction.x, 1.0f / ray.Direction.y, 1.0f / ray.Direction.z};
  for (uint k = 0; k < sc.nleaves && !th.end_search; ++k) {
    const uint l = sc.reverse ? sc.nleaves - 1 - k : k;
    const float *b = sc.boxes + 6 * (size_t)l;
    if (b[0] != b[0]) continue;  // inactive leaf (NaN box)
    bool hit;
    if (ray.TMin == ray.TMax) {  // a point query
      const float *o = &ray.Origin.x;
      hit = o[0] >= b[0] && o[0] <= b[3] && o[1] >= b[1] && o[1] <= b[4] && o[2] >= b[2] && o[2] <= b[5];
    } else {
      float tn = th.tmin, tf = th.tcur;
      for (int a = 0; a < 3; ++a) {
        const float o = (&ray.Origin.x)[a];
        float t0 = (b[a] - o) * inv[a], t1 = (b[3 + a] - o) * inv[a];
        if (t0 > t1) {
          const float s = t0;
          t0 = t1;
          t1 = s;
        }
        tn = fmaxf(tn, t0);
        tf = fminf(tf, t1);
      }
      hit = tn <= tf;
    }
    if (!hit) continue;
    th.primitive = l;
    href_intersection((int)ray_type);
  }
  const HrefThread inner = th;
  th = saved;
  (void)inner;
}

// ---- GPRT handles ------------------------------------------------------------------------------

struct Texture1D {
  const float *texels;  // n texels of `channels` floats
  int n, channels;
  float4 SampleGrad(SamplerState, float u, float, float) const {
    float v[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int c = 0; c < channels; ++c) v[c] = orc_tex_sample(texels, n, channels, c, u);
    return float4(v[0], v[1], v[2], v[3]);
  }
};

struct Texture2D {
  const float *texels;  // w x h texels of 4 floats, row-major
  int w, h;
  float4 fetch(int x, int y) const {
    x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
    y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
    const float *t = texels + 4 * ((size_t)y * (size_t)w + (size_t)x);
    return float4(t[0], t[1], t[2], t[3]);
  }
  float4 operator[](const uint2 &c) const { return fetch((int)c.x, (int)c.y); }
  float4 SampleGrad(SamplerState, const float2 &uv, const float2 &, const float2 &) const {
    const float fx = uv.x * (float)w - 0.5f, fy = uv.y * (float)h - 0.5f;
    const float x0 = floorf(fx), y0 = floorf(fy);
    const float ax = rintf((fx - x0) * 256.0f) / 256.0f, ay = rintf((fy - y0) * 256.0f) / 256.0f;
    const int ix = (int)x0, iy = (int)y0;
    const float4 t00 = fetch(ix, iy), t10 = fetch(ix + 1, iy), t01 = fetch(ix, iy + 1), t11 = fetch(ix + 1, iy + 1);
    if (ax == 0.0f && ay == 0.0f) return t00;
    if (ax == 1.0f && ay == 0.0f) return t10;
    if (ax == 0.0f && ay == 1.0f) return t01;
    if (ax == 1.0f && ay == 1.0f) return t11;
    const float4 top = t00 + ax * (t10 - t00), bot = t01 + ax * (t11 - t01);
    return top + ay * (bot - top);
  }
};

namespace gprt {
struct Buffer {
  void *p;
};
struct Texture {
  const void *p;
};
struct Accel {
  int unused;
};
inline RaytracingAccelerationStructure getAccelHandle(Accel) { return RaytracingAccelerationStructure{0}; }
inline SamplerState getDefaultSampler() { return SamplerState{0}; }
inline Texture1D getTexture1DHandle(Texture t) { return *static_cast<const Texture1D *>(t.p); }
inline Texture2D getTexture2DHandle(Texture t) { return *static_cast<const Texture2D *>(t.p); }
template <class T>
inline T load(Buffer b, uint i) {
  return static_cast<const T *>(b.p)[i];
}
template <class T>
inline void store(Buffer b, uint i, const T &v) {
  static_cast<T *>(b.p)[i] = v;
}
inline uint make_bgra(const float4 &c) {
  auto u8 = [](float v) { return (uint)(saturate(v) * 255.0f + 0.5f); };
  return u8(c.z) | (u8(c.y) << 8) | (u8(c.x) << 16) | (u8(c.w) << 24);
}
inline void ignoreHit() { href_thread().ignored = true; }
inline void acceptHitAndEndSearch() { href_thread().end_search = true; }
}  // namespace gprt

// ---- program declarations ---------------------------------------------------------------------------

#define HREF_IN(T, n) const T &n
#define HREF_INOUT(T, n) T &n
#define GPRT_RAYGEN_PROGRAM(name, rec) void name(HREF_IN rec)
#define GPRT_INTERSECTION_PROGRAM(name, rec) void name(HREF_IN rec)
#define GPRT_ANY_HIT_PROGRAM(name, rec, pay, attr) void name(HREF_IN rec, HREF_INOUT pay, HREF_IN attr)
#define GPRT_MISS_PROGRAM(name, rec, pay) void name(HREF_IN rec, HREF_INOUT pay)
#define GPRT_COMPUTE_PROGRAM(name, rec, dims) void name(HREF_IN rec)
