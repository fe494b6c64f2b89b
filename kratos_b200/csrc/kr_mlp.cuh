// Per-face HLLE/HLLD selector: a 16 -> 32 -> 32 -> 1 MLP (ReLU, logit out).
//
// Features (face_features) are 16 normalised left/right primitive-state
// combinations in the rotated frame; the training target is whether the HLLE
// flux of the face is within a tolerance of the HLLD flux (flux_gap).  The MLP
// is trained in FP32 by the hand-written kernels of kr_learn.cu and evaluated in
// the flux sweep with BF16 tensor-core MMAs (mma.sync m16n8k16, FP32
// accumulate): one warp evaluates its 32 faces together.
//
// No reference counterpart (the reference has HLLD only); parity of the
// selected step is judged against the all-HLLD FP64 step.
#pragma once

#include <cuda_bf16.h>
#include "kr_math.cuh"

namespace kr
{
constexpr int MLP_IN = 16, MLP_H = 32;
// parameter offsets in the flat FP32 vector (row-major W[in][out])
constexpr int MLP_W1 = 0;                                  // [16][32]
constexpr int MLP_B1 = MLP_W1 + MLP_IN * MLP_H;            // [32]
constexpr int MLP_W2 = MLP_B1 + MLP_H;                     // [32][32]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;             // [32]
constexpr int MLP_W3 = MLP_B2 + MLP_H;                     // [32]
constexpr int MLP_B3 = MLP_W3 + MLP_H;                     // [1]
constexpr int MLP_NPARAM = MLP_B3 + 1;                     // 1633

// Normalised features of a face from rotated primitive states (rho, p, vn,
// vt1, vt2, bn, bt1, bt2).
template< class R > __device__ __forceinline__
void face_features( const R * ql, const R * qr, R gamma, float * f )
{
    const float rl = float( ql[ RHO ] ), rr = float( qr[ RHO ] );
    const float pl = float( ql[ ENE ] ), pr = float( qr[ ENE ] );
    const float rb = 0.5f * ( rl + rr ), pb = 0.5f * ( pl + pr );
    float b2 = 0;
    for( int a = 0; a < 3; ++ a )
    {
        const float bm = 0.5f * float( ql[ BCC + a ] + qr[ BCC + a ] );
        b2 += bm * bm;
    }
    const float cs2 = float( gamma ) * pb / rb;
    const float cf  = sqrtf( cs2 + b2 / rb ) + 1e-30f;
    const float icf = 1.0f / cf;
    const float iva = icf * rsqrtf( rb );
    f[ 0 ] = ( rl - rr ) / rb;
    f[ 1 ] = ( pl - pr ) / pb;
    for( int a = 0; a < 3; ++ a )
    {
        f[ 2 + a ] = float( ql[ MOM + a ] - qr[ MOM + a ] ) * icf;
        f[ 5 + a ] = 0.5f * float( ql[ MOM + a ] + qr[ MOM + a ] ) * icf;
        f[ 10 + a ] = 0.5f * float( ql[ BCC + a ] + qr[ BCC + a ] ) * iva;
    }
    f[ 8 ] = float( ql[ BCC + 1 ] - qr[ BCC + 1 ] ) * iva;
    f[ 9 ] = float( ql[ BCC + 2 ] - qr[ BCC + 2 ] ) * iva;
    f[ 13 ] = sqrtf( cs2 ) * icf;
    f[ 14 ] = fabsf( f[ 0 ] );
    f[ 15 ] = fabsf( f[ 1 ] );
}

// Largest component of |F_hlle - F_hlld| in units of the face's flux scales
// (rho c, rho c^2, rho c^3, sqrt(rho) c^2 for mass, momentum, energy, EMF).
template< class R > __device__ __forceinline__
float flux_gap( const R * fe, const R * fd, const R * ql, const R * qr, R gamma )
{
    const double rb = 0.5 * double( ql[ RHO ] + qr[ RHO ] );
    const double pb = 0.5 * double( ql[ ENE ] + qr[ ENE ] );
    double b2 = 0;
    for( int a = 0; a < 3; ++ a )
    {
        const double bm = 0.5 * double( ql[ BCC + a ] + qr[ BCC + a ] );
        b2 += bm * bm;
    }
    const double c = sqrt( ( double( gamma ) * pb + b2 ) / rb );
    const double s[ 8 ] = { rb * c, rb * c * c * c, rb * c * c, rb * c * c, rb * c * c,
                            1, sqrt( rb ) * c * c, sqrt( rb ) * c * c };
    double g = 0;
    for( int k = 0; k < 8; ++ k )
        if( k != BCC )
            g = fmax( g, fabs( double( fe[ k ] ) - double( fd[ k ] ) ) / s[ k ] );
    return float( g );
}

////////////////////////////////////////////////////////////
// BF16 tensor-core inference: whole warp, one face per lane.
//
// `wb` holds the weights as bf16 in MMA-fragment order (mlp_pack_bf16), `bias`
// the FP32 biases, `xs` 32 x 16 bf16 of shared memory owned by this warp.
// Every lane of the warp must call this (mma.sync is warp-collective).

__device__ __forceinline__ unsigned pack_bf16( float a, float b )
{
    const __nv_bfloat162 v = __floats2bfloat162_rn( a, b );
    return * reinterpret_cast< const unsigned * >( & v );
}

__device__ __forceinline__ void mma_bf16( float * d, const unsigned * a, const unsigned * b )
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"( d[ 0 ] ), "+f"( d[ 1 ] ), "+f"( d[ 2 ] ), "+f"( d[ 3 ] )
        : "r"( a[ 0 ] ), "r"( a[ 1 ] ), "r"( a[ 2 ] ), "r"( a[ 3 ] ), "r"( b[ 0 ] ), "r"( b[ 1 ] ) );
}

// B-fragment words per layer: W1 4 n-tiles x 2 words; W2 4 n-tiles x 2 k-steps x
// 2 words; W3 (padded to 8 outputs) 2 k-steps x 2 words; per lane.
constexpr int MLP_BFRAG = ( 4 * 2 + 4 * 2 * 2 + 2 * 2 );   // 28 words per lane

// Weight words for lane `lane` in the order mlp_logit reads them (host and
// device use the same packing through this function).
__host__ __device__ inline void mlp_lane_words( const float * w, int lane, float * out56 )
{
    const int g = lane >> 2, t = lane & 3;
    int o = 0;
    // layer 1: k = 0..15, n-tile j: b0,b1 = W1[t*2+{0,1}][8j+g], b2,b3 = W1[t*2+8+{0,1}][8j+g]
    for( int j = 0; j < 4; ++ j )
    {
        out56[ o++ ] = w[ MLP_W1 + ( t * 2 + 0 ) * MLP_H + 8 * j + g ];
        out56[ o++ ] = w[ MLP_W1 + ( t * 2 + 1 ) * MLP_H + 8 * j + g ];
        out56[ o++ ] = w[ MLP_W1 + ( t * 2 + 8 ) * MLP_H + 8 * j + g ];
        out56[ o++ ] = w[ MLP_W1 + ( t * 2 + 9 ) * MLP_H + 8 * j + g ];
    }
    for( int j = 0; j < 4; ++ j )
        for( int s = 0; s < 2; ++ s )
        {
            out56[ o++ ] = w[ MLP_W2 + ( 16 * s + t * 2 + 0 ) * MLP_H + 8 * j + g ];
            out56[ o++ ] = w[ MLP_W2 + ( 16 * s + t * 2 + 1 ) * MLP_H + 8 * j + g ];
            out56[ o++ ] = w[ MLP_W2 + ( 16 * s + t * 2 + 8 ) * MLP_H + 8 * j + g ];
            out56[ o++ ] = w[ MLP_W2 + ( 16 * s + t * 2 + 9 ) * MLP_H + 8 * j + g ];
        }
    for( int s = 0; s < 2; ++ s )
    {   // output column 0 only (g == 0); other columns zero
        out56[ o++ ] = g == 0 ? w[ MLP_W3 + 16 * s + t * 2 + 0 ] : 0.f;
        out56[ o++ ] = g == 0 ? w[ MLP_W3 + 16 * s + t * 2 + 1 ] : 0.f;
        out56[ o++ ] = g == 0 ? w[ MLP_W3 + 16 * s + t * 2 + 8 ] : 0.f;
        out56[ o++ ] = g == 0 ? w[ MLP_W3 + 16 * s + t * 2 + 9 ] : 0.f;
    }
}

// Logit of this lane's face.  wpack: [32 lanes][28] bf16x2 words (device),
// bias: b1 (32), b2 (32), b3 (1) in FP32; xs: this warp's 32 x 16 bf16 scratch.
__device__ __forceinline__
float mlp_logit( const float * feat, const unsigned * wpack, const float * bias,
                 __nv_bfloat16 * xs )
{
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    for( int k = 0; k < MLP_IN; ++ k )
        xs[ lane * MLP_IN + k ] = __float2bfloat16_rn( feat[ k ] );
    __syncwarp(  );
    const unsigned * wl = wpack + lane * MLP_BFRAG;
    // layer 1: two m-tiles (faces 0..15, 16..31) x four n-tiles
    float h[ 2 ][ 4 ][ 4 ];
    for( int m = 0; m < 2; ++ m )
    {
        unsigned a[ 4 ];
        const __nv_bfloat16 * r0 = xs + ( 16 * m + g ) * MLP_IN;
        const __nv_bfloat16 * r1 = xs + ( 16 * m + g + 8 ) * MLP_IN;
        a[ 0 ] = * reinterpret_cast< const unsigned * >( r0 + t * 2 );
        a[ 1 ] = * reinterpret_cast< const unsigned * >( r1 + t * 2 );
        a[ 2 ] = * reinterpret_cast< const unsigned * >( r0 + t * 2 + 8 );
        a[ 3 ] = * reinterpret_cast< const unsigned * >( r1 + t * 2 + 8 );
        for( int j = 0; j < 4; ++ j )
        {
            for( int q = 0; q < 4; ++ q ) h[ m ][ j ][ q ] = 0.f;
            mma_bf16( h[ m ][ j ], a, wl + 2 * j );
        }
    }
    // bias + ReLU -> A fragments of layer 2 (accumulator layout maps onto them)
    float h2[ 2 ][ 4 ][ 4 ];
    for( int m = 0; m < 2; ++ m )
    {
        unsigned a[ 2 ][ 4 ];
        for( int s = 0; s < 2; ++ s )
        {
            const int j0 = 2 * s, j1 = 2 * s + 1;
            const float b00 = bias[ 8 * j0 + t * 2 ], b01 = bias[ 8 * j0 + t * 2 + 1 ];
            const float b10 = bias[ 8 * j1 + t * 2 ], b11 = bias[ 8 * j1 + t * 2 + 1 ];
            a[ s ][ 0 ] = pack_bf16( fmaxf( h[ m ][ j0 ][ 0 ] + b00, 0.f ), fmaxf( h[ m ][ j0 ][ 1 ] + b01, 0.f ) );
            a[ s ][ 1 ] = pack_bf16( fmaxf( h[ m ][ j0 ][ 2 ] + b00, 0.f ), fmaxf( h[ m ][ j0 ][ 3 ] + b01, 0.f ) );
            a[ s ][ 2 ] = pack_bf16( fmaxf( h[ m ][ j1 ][ 0 ] + b10, 0.f ), fmaxf( h[ m ][ j1 ][ 1 ] + b11, 0.f ) );
            a[ s ][ 3 ] = pack_bf16( fmaxf( h[ m ][ j1 ][ 2 ] + b10, 0.f ), fmaxf( h[ m ][ j1 ][ 3 ] + b11, 0.f ) );
        }
        for( int j = 0; j < 4; ++ j )
        {
            for( int q = 0; q < 4; ++ q ) h2[ m ][ j ][ q ] = 0.f;
            mma_bf16( h2[ m ][ j ], a[ 0 ], wl + 8 + 4 * j );
            mma_bf16( h2[ m ][ j ], a[ 1 ], wl + 8 + 4 * j + 2 );
        }
    }
    // layer 3 (output column 0)
    float z[ 2 ][ 4 ];
    for( int m = 0; m < 2; ++ m )
    {
        unsigned a[ 2 ][ 4 ];
        for( int s = 0; s < 2; ++ s )
        {
            const int j0 = 2 * s, j1 = 2 * s + 1;
            const float * b2 = bias + MLP_H;
            const float b00 = b2[ 8 * j0 + t * 2 ], b01 = b2[ 8 * j0 + t * 2 + 1 ];
            const float b10 = b2[ 8 * j1 + t * 2 ], b11 = b2[ 8 * j1 + t * 2 + 1 ];
            a[ s ][ 0 ] = pack_bf16( fmaxf( h2[ m ][ j0 ][ 0 ] + b00, 0.f ), fmaxf( h2[ m ][ j0 ][ 1 ] + b01, 0.f ) );
            a[ s ][ 1 ] = pack_bf16( fmaxf( h2[ m ][ j0 ][ 2 ] + b00, 0.f ), fmaxf( h2[ m ][ j0 ][ 3 ] + b01, 0.f ) );
            a[ s ][ 2 ] = pack_bf16( fmaxf( h2[ m ][ j1 ][ 0 ] + b10, 0.f ), fmaxf( h2[ m ][ j1 ][ 1 ] + b11, 0.f ) );
            a[ s ][ 3 ] = pack_bf16( fmaxf( h2[ m ][ j1 ][ 2 ] + b10, 0.f ), fmaxf( h2[ m ][ j1 ][ 3 ] + b11, 0.f ) );
        }
        for( int q = 0; q < 4; ++ q ) z[ m ][ q ] = 0.f;
        mma_bf16( z[ m ], a[ 0 ], wl + 24 );
        mma_bf16( z[ m ], a[ 1 ], wl + 26 );
    }
    // column 0 of row r sits in lane (r % 8) * 4: c0 for rows < 8, c2 for rows >= 8
    const int m = lane >> 4, r = lane & 15;
    const int src = ( r & 7 ) * 4;
    const float lo0 = __shfl_sync( 0xffffffffu, z[ 0 ][ 0 ], src );
    const float hi0 = __shfl_sync( 0xffffffffu, z[ 0 ][ 2 ], src );
    const float lo1 = __shfl_sync( 0xffffffffu, z[ 1 ][ 0 ], src );
    const float hi1 = __shfl_sync( 0xffffffffu, z[ 1 ][ 2 ], src );
    __syncwarp(  );
    const float v = m == 0 ? ( r < 8 ? lo0 : hi0 ) : ( r < 8 ? lo1 : hi1 );
    return v + bias[ 2 * MLP_H ];
}

}   // namespace kr
