// Training and standalone inference of the per-face HLLE/HLLD selector MLP
// (kr_mlp.cuh): hand-written FP32 forward / backward kernels with block-level
// gradient reduction, an Adam update kernel, and the BF16 tensor-core
// inference path exposed on its own for testing.
//
// Loss: class-weighted binary cross-entropy on the logit z,
//   l = w_y * ( max(z,0) - z y + log(1 + exp(-|z|)) ),  w_y = 1 (y=1), wneg (y=0),
// averaged over the samples.  y = 1 marks faces whose HLLE flux is within the
// tolerance of their HLLD flux ("safe"); wneg > 1 makes false "safe" calls cost
// more than missed ones.
#include "../../include/kratos_b200.h"
#include "kr_mlp.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace kr
{
constexpr int GRAD_SAMPLES = 64;     // samples per CTA in the gradient kernel
constexpr int GRAD_THREADS = 256;

// One CTA: forward / backward of GRAD_SAMPLES samples, then their summed
// contribution to every parameter gradient, written to the CTA's row of
// `partial` ([gridDim.x][MLP_NPARAM]); k_grad_sum adds the rows in a fixed
// order, so a gradient (and the training run) does not depend on the order
// in which CTAs finish.
__global__ void __launch_bounds__( GRAD_THREADS )
k_mlp_grad( const float * X, const float * Y, long long n0, long long n,
            const float * w, float wneg, float * partial, double * loss )
{
    __shared__ float sw[ MLP_NPARAM ];
    __shared__ float sx[ GRAD_SAMPLES ][ MLP_IN ];
    __shared__ float h1[ GRAD_SAMPLES ][ MLP_H ], h2[ GRAD_SAMPLES ][ MLP_H ];
    __shared__ float d1[ GRAD_SAMPLES ][ MLP_H ], d2[ GRAD_SAMPLES ][ MLP_H ];
    __shared__ float dz[ GRAD_SAMPLES ];
    __shared__ float sloss[ GRAD_SAMPLES ];
    for( int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x )
        sw[ k ] = w[ k ];
    const long long base = n0 + ( long long ) blockIdx.x * GRAD_SAMPLES;
    for( int k = threadIdx.x; k < GRAD_SAMPLES * MLP_IN; k += blockDim.x )
    {
        const int s = k / MLP_IN, i = k % MLP_IN;
        sx[ s ][ i ] = base + s < n ? X[ ( base + s ) * MLP_IN + i ] : 0.f;
    }
    __syncthreads(  );
    if( threadIdx.x < GRAD_SAMPLES )
    {
        const int s = threadIdx.x;
        const bool live = base + s < n;
        for( int j = 0; j < MLP_H; ++ j )
        {
            float a = sw[ MLP_B1 + j ];
            for( int i = 0; i < MLP_IN; ++ i )
                a += sx[ s ][ i ] * sw[ MLP_W1 + i * MLP_H + j ];
            h1[ s ][ j ] = fmaxf( a, 0.f );
        }
        for( int j = 0; j < MLP_H; ++ j )
        {
            float a = sw[ MLP_B2 + j ];
            for( int i = 0; i < MLP_H; ++ i )
                a += h1[ s ][ i ] * sw[ MLP_W2 + i * MLP_H + j ];
            h2[ s ][ j ] = fmaxf( a, 0.f );
        }
        float z = sw[ MLP_B3 ];
        for( int i = 0; i < MLP_H; ++ i )
            z += h2[ s ][ i ] * sw[ MLP_W3 + i ];
        const float y = live ? Y[ base + s ] : 0.f;
        const float wy = y > 0.5f ? 1.f : wneg;
        const float sig = 1.f / ( 1.f + expf( -z ) );
        const float g = live ? wy * ( sig - y ) : 0.f;
        dz[ s ] = g;
        sloss[ s ] = live ? wy * ( fmaxf( z, 0.f ) - z * y + log1pf( expf( -fabsf( z ) ) ) ) : 0.f;
        for( int i = 0; i < MLP_H; ++ i )
            d2[ s ][ i ] = h2[ s ][ i ] > 0.f ? g * sw[ MLP_W3 + i ] : 0.f;
        for( int i = 0; i < MLP_H; ++ i )
        {
            float a = 0.f;
            for( int j = 0; j < MLP_H; ++ j )
                a += sw[ MLP_W2 + i * MLP_H + j ] * d2[ s ][ j ];
            d1[ s ][ i ] = h1[ s ][ i ] > 0.f ? a : 0.f;
        }
    }
    __syncthreads(  );
    for( int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x )
    {
        float acc = 0.f;
        if( k < MLP_B1 )
        {
            const int i = k / MLP_H, j = k % MLP_H;
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += sx[ s ][ i ] * d1[ s ][ j ];
        }
        else if( k < MLP_W2 )
        {
            const int j = k - MLP_B1;
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += d1[ s ][ j ];
        }
        else if( k < MLP_B2 )
        {
            const int i = ( k - MLP_W2 ) / MLP_H, j = ( k - MLP_W2 ) % MLP_H;
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += h1[ s ][ i ] * d2[ s ][ j ];
        }
        else if( k < MLP_W3 )
        {
            const int j = k - MLP_B2;
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += d2[ s ][ j ];
        }
        else if( k < MLP_B3 )
        {
            const int i = k - MLP_W3;
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += h2[ s ][ i ] * dz[ s ];
        }
        else
            for( int s = 0; s < GRAD_SAMPLES; ++ s ) acc += dz[ s ];
        partial[ ( size_t ) blockIdx.x * MLP_NPARAM + k ] = acc;
    }
    if( threadIdx.x == 0 )
    {
        double l = 0;
        for( int s = 0; s < GRAD_SAMPLES; ++ s ) l += sloss[ s ];
        atomicAdd( loss, l );
    }
}

__global__ void k_grad_sum( const float * partial, int rows, float * grad )
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if( k >= MLP_NPARAM )
        return;
    float g = 0;
    for( int r = 0; r < rows; ++ r )
        g += partial[ ( size_t ) r * MLP_NPARAM + k ];
    grad[ k ] = g;
}

__global__ void k_adam( float * w, const float * grad, float * m, float * v, int t,
                        float lr, float inv_n )
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if( k >= MLP_NPARAM )
        return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float g = grad[ k ] * inv_n;
    m[ k ] = b1 * m[ k ] + ( 1 - b1 ) * g;
    v[ k ] = b2 * v[ k ] + ( 1 - b2 ) * g * g;
    const float mh = m[ k ] / ( 1 - powf( b1, float( t ) ) );
    const float vh = v[ k ] / ( 1 - powf( b2, float( t ) ) );
    w[ k ] -= lr * mh / ( sqrtf( vh ) + eps );
}

__global__ void k_mlp_infer( const float * X, long long n, const unsigned * wpack,
                             const float * bias, float * out )
{
    __shared__ __nv_bfloat16 xs[ 4 ][ 32 * MLP_IN ];
    const long long i = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    float f[ MLP_IN ];
    for( int k = 0; k < MLP_IN; ++ k )
        f[ k ] = i < n ? X[ i * MLP_IN + k ] : 0.f;
    const float z = mlp_logit( f, wpack, bias, xs[ threadIdx.x >> 5 ] );
    if( i < n )
        out[ i ] = z;
}

}   // namespace kr

using namespace kr;

static thread_local std::string g_learn_error;

static bool lk( cudaError_t e, const char * what )
{
    if( e == cudaSuccess ) return true;
    g_learn_error = std::string( what ) + ": " + cudaGetErrorString( e );
    return false;
}

// Host packing of the FP32 parameters into the per-lane bf16 fragment words
// and the FP32 bias vector used by mlp_logit.
void kr_mlp_pack( const float * w, std::vector< unsigned > & words, std::vector< float > & bias )
{
    words.resize( 32 * MLP_BFRAG );
    for( int lane = 0; lane < 32; ++ lane )
    {
        float v[ 2 * MLP_BFRAG ];
        mlp_lane_words( w, lane, v );
        for( int q = 0; q < MLP_BFRAG; ++ q )
        {
            const __nv_bfloat162 p = __floats2bfloat162_rn( v[ 2 * q ], v[ 2 * q + 1 ] );
            words[ lane * MLP_BFRAG + q ] = * reinterpret_cast< const unsigned * >( & p );
        }
    }
    bias.assign( w + MLP_B1, w + MLP_B1 + MLP_H );
    bias.insert( bias.end(  ), w + MLP_B2, w + MLP_B2 + MLP_H );
    bias.push_back( w[ MLP_B3 ] );
}

extern "C" {

const char * kr_learn_last_error( void ) { return g_learn_error.c_str(  ); }

int kr_mlp_param_count( void ) { return MLP_NPARAM; }

void kr_mlp_init( float * w, uint64_t seed )
{
    std::mt19937_64 rng( seed );
    std::normal_distribution< float > nd( 0.f, 1.f );
    for( int k = 0; k < MLP_NPARAM; ++ k ) w[ k ] = 0.f;
    for( int k = MLP_W1; k < MLP_B1; ++ k ) w[ k ] = nd( rng ) * sqrtf( 2.f / MLP_IN );
    for( int k = MLP_W2; k < MLP_B2; ++ k ) w[ k ] = nd( rng ) * sqrtf( 2.f / MLP_H );
    for( int k = MLP_W3; k < MLP_B3; ++ k ) w[ k ] = nd( rng ) * sqrtf( 1.f / MLP_H );
}

// Mean loss and mean gradient of the selector MLP over n samples (one pass of
// the training kernels; for checking them against a CPU restatement).
int kr_mlp_grad( const float * X, const float * Y, long long n, const float * w, float wneg,
                 float * grad_out, double * loss_out, int device )
{
    g_learn_error.clear(  );
    if( ! X || ! Y || ! w || ! grad_out || n <= 0 ) { g_learn_error = "kr_mlp_grad: bad arguments"; return -1; }
    if( ! lk( cudaSetDevice( device ), "cudaSetDevice" ) ) return -1;
    float * dX = nullptr, * dY = nullptr, * dw = nullptr, * dg = nullptr, * dp = nullptr;
    double * dl = nullptr;
    const unsigned nb = unsigned( ( n + GRAD_SAMPLES - 1 ) / GRAD_SAMPLES );
    bool ok = lk( cudaMalloc( & dX, n * MLP_IN * 4 ), "malloc" ) && lk( cudaMalloc( & dY, n * 4 ), "malloc" )
           && lk( cudaMalloc( & dw, MLP_NPARAM * 4 ), "malloc" ) && lk( cudaMalloc( & dg, MLP_NPARAM * 4 ), "malloc" )
           && lk( cudaMalloc( & dp, size_t( nb ) * MLP_NPARAM * 4 ), "malloc" ) && lk( cudaMalloc( & dl, 8 ), "malloc" );
    ok = ok && lk( cudaMemcpy( dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( dY, Y, n * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( dw, w, MLP_NPARAM * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemset( dg, 0, MLP_NPARAM * 4 ), "memset" ) && lk( cudaMemset( dl, 0, 8 ), "memset" );
    if( ok )
    {
        k_mlp_grad<<< nb, GRAD_THREADS >>>( dX, dY, 0, n, dw, wneg, dp, dl );
        k_grad_sum<<< ( MLP_NPARAM + 255 ) / 256, 256 >>>( dp, int( nb ), dg );
        ok = lk( cudaGetLastError(  ), "k_mlp_grad" ) && lk( cudaDeviceSynchronize(  ), "sync" );
    }
    double l = 0;
    ok = ok && lk( cudaMemcpy( grad_out, dg, MLP_NPARAM * 4, cudaMemcpyDeviceToHost ), "download" )
            && lk( cudaMemcpy( & l, dl, 8, cudaMemcpyDeviceToHost ), "download" );
    if( ok )
    {
        for( int k = 0; k < MLP_NPARAM; ++ k ) grad_out[ k ] /= float( n );
        if( loss_out ) * loss_out = l / double( n );
    }
    cudaFree( dX ); cudaFree( dY ); cudaFree( dw ); cudaFree( dg ); cudaFree( dp ); cudaFree( dl );
    return ok ? 0 : -1;
}

// Adam training on the GPU.  w: in/out FP32 parameters (kr_mlp_init for a fresh
// network).  Mini-batches are consecutive slices of the (caller-shuffled) data.
int kr_mlp_train( const float * X, const float * Y, long long n, float * w, int epochs,
                  int batch, float lr, float wneg, double * loss_out, int device )
{
    g_learn_error.clear(  );
    if( ! X || ! Y || ! w || n <= 0 || epochs <= 0 || batch <= 0 )
    {
        g_learn_error = "kr_mlp_train: bad arguments";
        return -1;
    }
    if( ! lk( cudaSetDevice( device ), "cudaSetDevice" ) ) return -1;
    float * dX = nullptr, * dY = nullptr, * dw = nullptr, * dg = nullptr, * dm = nullptr, * dv = nullptr;
    float * dp = nullptr;
    double * dl = nullptr;
    const long long rows = ( std::min( n, ( long long ) batch ) + GRAD_SAMPLES - 1 ) / GRAD_SAMPLES;
    bool ok = lk( cudaMalloc( & dX, n * MLP_IN * 4 ), "malloc" ) && lk( cudaMalloc( & dY, n * 4 ), "malloc" )
           && lk( cudaMalloc( & dw, MLP_NPARAM * 4 ), "malloc" ) && lk( cudaMalloc( & dg, MLP_NPARAM * 4 ), "malloc" )
           && lk( cudaMalloc( & dm, MLP_NPARAM * 4 ), "malloc" ) && lk( cudaMalloc( & dv, MLP_NPARAM * 4 ), "malloc" )
           && lk( cudaMalloc( & dp, size_t( rows ) * MLP_NPARAM * 4 ), "malloc" ) && lk( cudaMalloc( & dl, 8 ), "malloc" );
    ok = ok && lk( cudaMemcpy( dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( dY, Y, n * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( dw, w, MLP_NPARAM * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemset( dm, 0, MLP_NPARAM * 4 ), "memset" ) && lk( cudaMemset( dv, 0, MLP_NPARAM * 4 ), "memset" );
    int t = 0;
    double last = 0;
    for( int e = 0; e < epochs && ok; ++ e )
    {
        cudaMemset( dl, 0, 8 );
        for( long long b0 = 0; b0 < n && ok; b0 += batch )
        {
            const long long b1 = std::min( n, b0 + ( long long ) batch );
            const unsigned nb = unsigned( ( b1 - b0 + GRAD_SAMPLES - 1 ) / GRAD_SAMPLES );
            k_mlp_grad<<< nb, GRAD_THREADS >>>( dX, dY, b0, b1, dw, wneg, dp, dl );
            k_grad_sum<<< ( MLP_NPARAM + 255 ) / 256, 256 >>>( dp, int( nb ), dg );
            k_adam<<< ( MLP_NPARAM + 255 ) / 256, 256 >>>( dw, dg, dm, dv, ++ t, lr, 1.f / float( b1 - b0 ) );
            ok = lk( cudaGetLastError(  ), "train kernels" );
        }
        double l = 0;
        ok = ok && lk( cudaMemcpy( & l, dl, 8, cudaMemcpyDeviceToHost ), "download" );
        last = l / double( n );
    }
    ok = ok && lk( cudaMemcpy( w, dw, MLP_NPARAM * 4, cudaMemcpyDeviceToHost ), "download" );
    if( ok && loss_out ) * loss_out = last;
    cudaFree( dX ); cudaFree( dY ); cudaFree( dw ); cudaFree( dg ); cudaFree( dm ); cudaFree( dv );
    cudaFree( dp ); cudaFree( dl );
    return ok ? 0 : -1;
}

// Logits of n feature vectors through the BF16 tensor-core path of the flux sweep.
int kr_mlp_infer( const float * X, long long n, const float * w, float * logit_out, int device )
{
    g_learn_error.clear(  );
    if( ! X || ! w || ! logit_out || n <= 0 ) { g_learn_error = "kr_mlp_infer: bad arguments"; return -1; }
    if( ! lk( cudaSetDevice( device ), "cudaSetDevice" ) ) return -1;
    std::vector< unsigned > words;
    std::vector< float > bias;
    kr_mlp_pack( w, words, bias );
    float * dX = nullptr, * dO = nullptr, * db = nullptr;
    unsigned * dw = nullptr;
    bool ok = lk( cudaMalloc( & dX, n * MLP_IN * 4 ), "malloc" ) && lk( cudaMalloc( & dO, n * 4 ), "malloc" )
           && lk( cudaMalloc( & dw, words.size(  ) * 4 ), "malloc" ) && lk( cudaMalloc( & db, bias.size(  ) * 4 ), "malloc" );
    ok = ok && lk( cudaMemcpy( dX, X, n * MLP_IN * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( dw, words.data(  ), words.size(  ) * 4, cudaMemcpyHostToDevice ), "upload" )
            && lk( cudaMemcpy( db, bias.data(  ), bias.size(  ) * 4, cudaMemcpyHostToDevice ), "upload" );
    if( ok )
    {
        k_mlp_infer<<< unsigned( ( n + 127 ) / 128 ), 128 >>>( dX, n, dw, db, dO );
        ok = lk( cudaGetLastError(  ), "k_mlp_infer" ) && lk( cudaDeviceSynchronize(  ), "sync" );
    }
    ok = ok && lk( cudaMemcpy( logit_out, dO, n * 4, cudaMemcpyDeviceToHost ), "download" );
    cudaFree( dX ); cudaFree( dO ); cudaFree( dw ); cudaFree( db );
    return ok ? 0 : -1;
}

}   // extern "C"
