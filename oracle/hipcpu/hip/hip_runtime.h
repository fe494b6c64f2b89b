// Project-written HIP-CPU-compatible runtime header.
//
// Test infrastructure only: it lets the reference's own ARCH=HIPCPU code path
// (Makefile:40-55 of the reference, `-include hip/hip_runtime.h`) compile with
// plain g++ in a machine that has neither ROCm's HIP-CPU library nor TBB.  It is
// used to build the reference solver into oracle/_ref/ as a CPU oracle and as the
// timed CPU baseline; nothing in the product links it.
//
// Execution model.  A kernel launch runs to completion before the call returns
// (every stream is synchronous).  Blocks of a grid are distributed over a pool
// of host threads (KR_REF_THREADS, default: all hardware threads); the threads of one block run one after another on the same OS thread.
// That is exact for kernels whose threads never meet at __syncthreads().  The
// reference's cooperative kernels (flux_kernel, c2p, the comm packs) size their
// blocks from `[dynamics] thread_limit` / `bnd_thread_limit`; the recipe under
// oracle/ sets both to 1, so those blocks hold one thread and every barrier is
// trivially satisfied.  __syncthreads() aborts if it is ever reached by a block of
// more than one thread, so a silent mis-execution cannot happen.
#pragma once

#ifndef __HIPCC__
#define __HIPCC__ 1
#endif
#ifndef __HIP_CPU_RT__
#define __HIP_CPU_RT__ 1
#endif

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <functional>
#include <vector>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <type_traits>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__
#ifndef __forceinline__
#define __forceinline__ inline
#endif

struct dim3
{
    unsigned x, y, z;
    constexpr dim3( unsigned x_ = 1, unsigned y_ = 1, unsigned z_ = 1 )
        : x( x_ ), y( y_ ), z( z_ ) {}
};

inline thread_local dim3 threadIdx( 0, 0, 0 );
inline thread_local dim3 blockIdx ( 0, 0, 0 );
inline thread_local dim3 blockDim ( 1, 1, 1 );
inline thread_local dim3 gridDim  ( 1, 1, 1 );

namespace hipcpu
{
inline thread_local std::vector< char > smem;      // dynamic shared memory of the running block
inline char * dyn_smem(  ) { return smem.data(  ); }
}

#define HIP_DYNAMIC_SHARED( type, var ) \
    type * var = reinterpret_cast< type * >( hipcpu::dyn_smem(  ) )

inline void __syncthreads(  )
{
    if( blockDim.x * blockDim.y * blockDim.z > 1 )
    {
        std::fprintf( stderr, "hipcpu: __syncthreads() in a block of %u threads;"
                      " set [dynamics] thread_limit = bnd_thread_limit = 1\n",
                      blockDim.x * blockDim.y * blockDim.z );
        std::abort(  );
    }
}

////////////////////////////////////////////////////////////
// Types and error codes

enum hipError_t { hipSuccess = 0, hipErrorInvalidValue = 1, hipErrorMemoryAllocation = 2 };
enum hipMemcpyKind { hipMemcpyHostToHost = 0, hipMemcpyHostToDevice = 1,
                     hipMemcpyDeviceToHost = 2, hipMemcpyDeviceToDevice = 3,
                     hipMemcpyDefault = 4 };
enum hipFuncCache_t { hipFuncCachePreferNone = 0, hipFuncCachePreferShared = 1,
                      hipFuncCachePreferL1 = 2, hipFuncCachePreferEqual = 3 };
enum hipSharedMemConfig { hipSharedMemBankSizeDefault = 0,
                          hipSharedMemBankSizeFourByte = 1,
                          hipSharedMemBankSizeEightByte = 2 };
enum { hipHostRegisterDefault = 0 };

struct hipcpu_stream_s { int id; };
struct hipcpu_event_s  { int id; };
typedef hipcpu_stream_s * hipStream_t;
typedef hipcpu_event_s  * hipEvent_t;
typedef void ( * hipHostFn_t )( void * );

inline const char * hipGetErrorString( hipError_t e )
{
    return e == hipSuccess ? "hipSuccess" : "hipcpu error";
}

////////////////////////////////////////////////////////////
// Device and memory

inline hipError_t hipSetDevice( int ) { return hipSuccess; }
inline hipError_t hipGetDeviceCount( int * n ) { * n = 1; return hipSuccess; }
inline hipError_t hipDeviceSynchronize(  ) { return hipSuccess; }
inline hipError_t hipDeviceReset(  ) { return hipSuccess; }
inline hipError_t hipDeviceSetCacheConfig( hipFuncCache_t ) { return hipSuccess; }
inline hipError_t hipDeviceSetSharedMemConfig( hipSharedMemConfig ) { return hipSuccess; }

inline hipError_t hipMalloc( void ** p, size_t n )
{
    * p = std::aligned_alloc( 256, ( n + 255 ) / 256 * 256 + 256 );
    return * p ? hipSuccess : hipErrorMemoryAllocation;
}
template< class T > inline hipError_t hipMalloc( T ** p, size_t n )
{
    return hipMalloc( reinterpret_cast< void ** >( p ), n );
}
inline hipError_t hipHostMalloc( void ** p, size_t n, unsigned = 0 )
{
    return hipMalloc( p, n );
}
template< class T > inline hipError_t hipHostMalloc( T ** p, size_t n, unsigned f = 0 )
{
    return hipHostMalloc( reinterpret_cast< void ** >( p ), n, f );
}
inline hipError_t hipFree    ( void * p ) { std::free( p ); return hipSuccess; }
inline hipError_t hipHostFree( void * p ) { std::free( p ); return hipSuccess; }
inline hipError_t hipHostRegister( void *, size_t, unsigned ) { return hipSuccess; }
inline hipError_t hipHostUnregister( void * ) { return hipSuccess; }

inline hipError_t hipMemcpy( void * t, const void * s, size_t n, hipMemcpyKind )
{
    if( n ) std::memmove( t, s, n );
    return hipSuccess;
}
inline hipError_t hipMemcpyAsync( void * t, const void * s, size_t n,
                                  hipMemcpyKind k, hipStream_t = nullptr )
{
    return hipMemcpy( t, s, n, k );
}
inline hipError_t hipMemset( void * p, int v, size_t n )
{
    if( n ) std::memset( p, v, n );
    return hipSuccess;
}
inline hipError_t hipMemsetAsync( void * p, int v, size_t n, hipStream_t = nullptr )
{
    return hipMemset( p, v, n );
}
inline hipError_t hipMemcpyToSymbol( const void * sym, const void * src, size_t n,
                                     size_t offset = 0,
                                     hipMemcpyKind = hipMemcpyHostToDevice )
{
    std::memcpy( ( char * ) sym + offset, src, n );
    return hipSuccess;
}
template< class T >
inline hipError_t hipGetSymbolAddress( void ** p, const T & sym )
{
    * p = ( void * ) & sym;
    return hipSuccess;
}

////////////////////////////////////////////////////////////
// Streams and events: execution is synchronous, so they only need identities.

inline hipError_t hipStreamCreate( hipStream_t * s )
{
    * s = new hipcpu_stream_s{ 0 };
    return hipSuccess;
}
inline hipError_t hipStreamDestroy( hipStream_t s ) { delete s; return hipSuccess; }
inline hipError_t hipStreamSynchronize( hipStream_t ) { return hipSuccess; }
inline hipError_t hipStreamWaitEvent( hipStream_t, hipEvent_t, unsigned ) { return hipSuccess; }
inline hipError_t hipEventCreate( hipEvent_t * e )
{
    * e = new hipcpu_event_s{ 0 };
    return hipSuccess;
}
inline hipError_t hipEventDestroy( hipEvent_t e ) { delete e; return hipSuccess; }
inline hipError_t hipEventRecord( hipEvent_t, hipStream_t = nullptr ) { return hipSuccess; }
inline hipError_t hipEventSynchronize( hipEvent_t ) { return hipSuccess; }
inline hipError_t hipLaunchHostFunc( hipStream_t, hipHostFn_t f, void * p )
{
    f( p );
    return hipSuccess;
}

////////////////////////////////////////////////////////////
// Kernel launch: blocks over OpenMP threads, threads of a block in sequence.

namespace hipcpu
{
// Persistent worker pool: a launch hands out blocks through an atomic counter;
// the calling thread works too and returns when every block has finished and
// every worker has checked in for this launch.
struct pool_t
{
    std::vector< std::thread >  workers;
    std::mutex                  mtx;
    std::condition_variable     cv;
    const std::function< void( long long ) > * job = nullptr;
    long long                   n_jobs  = 0;
    std::atomic< long long >    next { 0 };
    std::atomic< long long >    done { 0 };
    std::atomic< long long >    left { 0 };   // workers finished with this launch
    unsigned long long          epoch   = 0;
    bool                        quit    = false;

    pool_t(  )
    {
        unsigned n = std::thread::hardware_concurrency(  );
        if( const char * e = std::getenv( "KR_REF_THREADS" ) )
            n = unsigned( std::atoi( e ) );
        n = std::max( 1u, n );
        for( unsigned t = 1; t < n; ++ t )
            workers.emplace_back( [ this ] (  ) { loop(  ); } );
    }
    ~pool_t(  )
    {
        { std::lock_guard< std::mutex > l( mtx ); quit = true; }
        cv.notify_all(  );
        for( auto & w : workers ) w.join(  );
    }
    void work(  )
    {
        for( ;; )
        {
            const long long b = next.fetch_add( 1 );
            if( b >= n_jobs ) break;
            ( * job )( b );
            done.fetch_add( 1 );
        }
    }
    void loop(  )
    {
        unsigned long long seen = 0;
        for( ;; )
        {
            {
                std::unique_lock< std::mutex > l( mtx );
                cv.wait( l, [ & ] { return quit || epoch != seen; } );
                if( quit ) return;
                seen = epoch;
            }
            work(  );
            left.fetch_add( 1 );
        }
    }
    void run( long long n, const std::function< void( long long ) > & f )
    {
        if( n <= 0 ) return;
        if( workers.empty(  ) || n == 1 )
        {
            for( long long b = 0; b < n; ++ b ) f( b );
            return;
        }
        {
            std::lock_guard< std::mutex > l( mtx );
            job = & f; n_jobs = n; next = 0; done = 0; left = 0; ++ epoch;
        }
        cv.notify_all(  );
        work(  );
        // Every worker must have left work() before the next launch resets the
        // counters, or a late worker could pick up a block index of this one.
        while( done.load(  ) < n || left.load(  ) < ( long long ) workers.size(  ) )
            std::this_thread::yield(  );
    }
};
inline pool_t & pool(  ) { static pool_t p; return p; }
}   // namespace hipcpu

inline void hipLaunchKernelGGL( const std::function< void(  ) > & ker,
                                const dim3 & n_bl, const dim3 & n_th,
                                int s_sh, hipStream_t = nullptr )
{
    const long long nbx = n_bl.x, nby = n_bl.y, nbz = n_bl.z;
    const std::function< void( long long ) > one_block = [ & ] ( long long b )
    {
        hipcpu::smem.resize( std::max( s_sh, 1 ) + 64 );
        gridDim  = n_bl;
        blockDim = n_th;
        blockIdx = dim3( unsigned( b % nbx ), unsigned( ( b / nbx ) % nby ),
                         unsigned( b / ( nbx * nby ) ) );
        for( unsigned tz = 0; tz < n_th.z; ++ tz )
            for( unsigned ty = 0; ty < n_th.y; ++ ty )
                for( unsigned tx = 0; tx < n_th.x; ++ tx )
                {
                    threadIdx = dim3( tx, ty, tz );
                    ker(  );
                }
    };
    hipcpu::pool(  ).run( nbx * nby * nbz, one_block );
}

////////////////////////////////////////////////////////////
// Atomics (host memory, GCC builtins)

inline int atomicCAS( int * p, int cmp, int val )
{
    __atomic_compare_exchange_n( p, & cmp, val, false,
                                 __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST );
    return cmp;
}
inline unsigned atomicCAS( unsigned * p, unsigned cmp, unsigned val )
{
    __atomic_compare_exchange_n( p, & cmp, val, false,
                                 __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST );
    return cmp;
}
inline unsigned long long atomicCAS( unsigned long long * p,
                                     unsigned long long cmp,
                                     unsigned long long val )
{
    __atomic_compare_exchange_n( p, & cmp, val, false,
                                 __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST );
    return cmp;
}
template< class T > inline T atomicAdd( T * p, T v )
{
    if constexpr( std::is_integral_v< T > )
        return __atomic_fetch_add( p, v, __ATOMIC_SEQ_CST );
    else
    {
        T old = * p, nxt;
        do { nxt = old + v; }
        while( ! __atomic_compare_exchange( p, & old, & nxt, false,
                                            __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST ) );
        return old;
    }
}
template< class T > inline T atomicExch( T * p, T v )
{
    return __atomic_exchange_n( p, v, __ATOMIC_SEQ_CST );
}
template< class T > inline T atomicMax( T * p, T v )
{
    T old = * p;
    while( old < v && ! __atomic_compare_exchange_n( p, & old, v, false,
                                                     __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST ) ) {}
    return old;
}
template< class T > inline T atomicMin( T * p, T v )
{
    T old = * p;
    while( old > v && ! __atomic_compare_exchange_n( p, & old, v, false,
                                                     __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST ) ) {}
    return old;
}

////////////////////////////////////////////////////////////
// Bit casts and math intrinsics not provided by the reference's own
// device_macros.h for the HIP-CPU mode.

inline double __longlong_as_double( long long x )
{
    double t;
    std::memcpy( & t, & x, sizeof( t ) );
    return t;
}
inline double __dsqrt_rn( double x ) { return std::sqrt( x ); }
inline float  __fsqrt_rn( float  x ) { return std::sqrt( x ); }
inline float  __powf( float a, float b ) { return std::pow( a, b ); }
inline float  __expf( float a ) { return std::exp( a ); }
inline float  __sinf( float a ) { return std::sin( a ); }
inline float  __cosf( float a ) { return std::cos( a ); }
inline float  __logf( float a ) { return std::log( a ); }
using std::fmaxf;
using std::fminf;
