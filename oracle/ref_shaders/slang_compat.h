/*
 * slang_compat.h - the HLSL/Slang subset the reference's per-thread raster
 * shaders use, as plain C++, so those shader files compile unchanged (after
 * the attribute/semantic strip in build_ref.sh) into a host library.
 *
 * TEST INFRASTRUCTURE ONLY: the result pins the oracle's restatement of the
 * shader arithmetic to the reference's own source.
 *
 * Semantics chosen where Slang/SPIR-V leaves them to the driver:
 *   dot(a, b)        (a.x*b.x + a.y*b.y) + a.z*b.z, no FMA (-ffp-contract=off)
 *   exp              vox_expf_cr (double-evaluated, correctly rounded in all
 *                    but tie cases, hence monotone: the 64-sample maximum of
 *                    gaussian_frag_color.slang:190-197 is attained at the
 *                    sample of least squared distance)
 *   log / pow        vox_logf / vox_powf (vox_detmath.h)
 *   sqrt             IEEE sqrtf
 * These are the same definitions the oracle and the CUDA kernels use.
 *
 * Include this header INSIDE the namespace that wraps one shader so that the
 * exp/log/pow/min/max overloads here hide the C library's.
 */
typedef uint32_t uint;

struct uint2
{
    uint x, y;
    uint2() : x(0u), y(0u) {}
    uint2(uint a, uint b) : x(a), y(b) {}
};
struct uint3
{
    uint x, y, z;
    uint3() : x(0u), y(0u), z(0u) {}
    uint3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
};
struct uint4
{
    uint x, y, z, w;
    uint4() : x(0u), y(0u), z(0u), w(0u) {}
    uint4(uint a, uint b, uint c, uint d) : x(a), y(b), z(c), w(d) {}
};
struct bool3
{
    bool x, y, z;
};

struct int3;
struct float3
{
    float x, y, z;
    float3() : x(0.f), y(0.f), z(0.f) {}
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit float3(float a) : x(a), y(a), z(a) {}
    explicit float3(const int3& v);
    float3& operator+=(const float3& o)
    {
        x = x + o.x;
        y = y + o.y;
        z = z + o.z;
        return *this;
    }
    float3& operator-=(const float3& o)
    {
        x = x - o.x;
        y = y - o.y;
        z = z - o.z;
        return *this;
    }
    float3& operator*=(const float3& o)
    {
        x = x * o.x;
        y = y * o.y;
        z = z * o.z;
        return *this;
    }
    float3& operator*=(float s)
    {
        x = x * s;
        y = y * s;
        z = z * s;
        return *this;
    }
};
struct int3
{
    int x, y, z;
    int3() : x(0), y(0), z(0) {}
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit int3(const float3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
    int3& operator+=(const int3& o)
    {
        x += o.x;
        y += o.y;
        z += o.z;
        return *this;
    }
};
inline float3::float3(const int3& v) : x((float)v.x), y((float)v.y), z((float)v.z) {}

struct float4
{
    union
    {
        struct
        {
            float x, y, z, w;
        };
        struct
        {
            float r, g, b, a;
        };
    };
    float4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    float4(float a0, float a1, float a2, float a3) : x(a0), y(a1), z(a2), w(a3) {}
    float4(const float3& v, float a3) : x(v.x), y(v.y), z(v.z), w(a3) {}
    /* the `.xyz` swizzle, spelled `.xyz()` by build_ref.sh */
    float3 xyz() const
    {
        return float3(x, y, z);
    }
};

/* float4x4 as the shader indexes it, m[row][column].  mul(v, M) treats v as a
 * row vector: result_j = ((v.x M[0][j] + v.y M[1][j]) + v.z M[2][j]) + v.w M[3][j]. */
struct float4x4
{
    float m[4][4];
};
inline float4 mul(const float4& v, const float4x4& M)
{
    float r[4];
    for (int j = 0; j < 4; j++)
    {
        float s = v.x * M.m[0][j] + v.y * M.m[1][j];
        s = s + v.z * M.m[2][j];
        r[j] = s + v.w * M.m[3][j];
    }
    return float4(r[0], r[1], r[2], r[3]);
}

inline float3 operator*(const float3& a, const float3& b)
{
    return float3(a.x * b.x, a.y * b.y, a.z * b.z);
}
inline float3 operator*(float s, const float3& b)
{
    return float3(s * b.x, s * b.y, s * b.z);
}
inline float3 operator*(const float3& a, float s)
{
    return float3(a.x * s, a.y * s, a.z * s);
}
inline float3 operator/(const float3& a, const float3& b)
{
    return float3(a.x / b.x, a.y / b.y, a.z / b.z);
}
inline float3 operator+(const float3& a, const float3& b)
{
    return float3(a.x + b.x, a.y + b.y, a.z + b.z);
}
inline float3 operator-(float s, const float3& b)
{
    return float3(s - b.x, s - b.y, s - b.z);
}
inline float3 operator-(const float3& a, const float3& b)
{
    return float3(a.x - b.x, a.y - b.y, a.z - b.z);
}
inline float3 operator-(const float3& a)
{
    return float3(-a.x, -a.y, -a.z);
}
inline float3 operator+(const float3& a, float s)
{
    return float3(a.x + s, a.y + s, a.z + s);
}
inline float3 operator/(const float3& a, float s)
{
    return float3(a.x / s, a.y / s, a.z / s);
}
inline int3 operator&(const int3& a, int m)
{
    return int3(a.x & m, a.y & m, a.z & m);
}
inline float3 floor(const float3& a)
{
    return float3(floorf(a.x), floorf(a.y), floorf(a.z));
}
inline int3 operator+(const int3& a, int s)
{
    return int3(a.x + s, a.y + s, a.z + s);
}
inline int3 operator-(const int3& a, const int3& b)
{
    return int3(a.x - b.x, a.y - b.y, a.z - b.z);
}

inline float min(float a, float b)
{
    return a < b ? a : b;
}
inline float max(float a, float b)
{
    return a > b ? a : b;
}
inline float3 min(const float3& a, const float3& b)
{
    return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
inline float3 max(const float3& a, const float3& b)
{
    return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
inline int3 min(const int3& a, const int3& b)
{
    return int3(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z);
}
inline int3 max(const int3& a, const int3& b)
{
    return int3(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z);
}
inline float dot(const float3& a, const float3& b)
{
    float xy = a.x * b.x + a.y * b.y;
    return xy + a.z * b.z;
}
inline float length(const float3& a)
{
    return sqrtf(dot(a, a));
}
inline float floor(float a)
{
    return floorf(a);
}
inline float sqrt(float a)
{
    return sqrtf(a);
}
inline float exp(float a)
{
    return vox_expf_cr(a);
}
inline float log(float a)
{
    return vox_logf(a);
}
inline float pow(float b, float e)
{
    return vox_powf(b, e);
}
inline float asfloat(uint u)
{
    return vox_u2f(u);
}
inline void InterlockedMax(uint& dst, uint v)
{
    dst = v > dst ? v : dst;
}

template <class T>
struct StructuredBuffer
{
    T* p;
    T& operator[](uint64_t i) const
    {
        return p[i];
    }
};
template <class T>
using RWStructuredBuffer = StructuredBuffer<T>;
template <class T>
using ConstantBuffer = T;
