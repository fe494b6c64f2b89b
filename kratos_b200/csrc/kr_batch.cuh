// Batched launch over blocks of uneven sizes: the size groups of a batch of
// independent periodic boxes (KR_FLAG_BOXES contexts, one per edge length).
//
// Every kernel kind of the step runs as ONE persistent launch whose CTAs walk
// a work list: one item per CTA tile that the per-group launches would run
// (group, block, z plane, tile along the plane), bigger blocks first.  A CTA
// takes items blockIdx.x, blockIdx.x + gridDim.x, ... and runs the same
// per-site code on the item's group arguments (read from the kernel's
// parameter space by the item's group index), so a batched step gives the
// per-group steps' results bit for bit while 1024 boxes of five sizes step in
// 14 launches instead of 5 x 14, captured as one CUDA graph.  The list is not
// stored: an item is decoded from its number with the list's per-group
// offsets and extents (batch_item), so the group index -- and every argument
// read through it -- is the same for all threads of the CTA and the compiler
// can keep it in uniform registers.  The number of resident CTAs of each
// launch is a tuning parameter (kr_batch_autotune).
//
// Included at the end of kr_core.cu (it uses the engine's kernels' device
// functions and the context internals).

namespace kr
{
constexpr int KR_BATCH_MAX = 6;

template< class R >
struct multi_t
{
    args_t< R > a[ KR_BATCH_MAX ];
    udiv_t dv_c[ KR_BATCH_MAX ];          // c2p rows: n0
    udiv_t dv_e[ KR_BATCH_MAX ];          // edge / lattice rows: n0 + 1
    udiv_t dv_f[ 3 ][ KR_BATCH_MAX ];     // face rows of each sweep
    unsigned cpp_f[ 3 ][ KR_BATCH_MAX ];  // 128-face tiles per z plane of each sweep
    // the work lists [c2p | flux z | flux y | flux x | lattice sites]: per list,
    // the first item of each group in list order (l_off[.][ng] = the count),
    // that group, and its tiles per plane and planes per block
    int ng;
    int l_off[ 5 ][ KR_BATCH_MAX + 1 ];
    int l_grp[ 5 ][ KR_BATCH_MAX ];
    udiv_t l_tiles[ 5 ][ KR_BATCH_MAX ];   // multiply-high quotients (d = 1: the identity)
    udiv_t l_planes[ 5 ][ KR_BATCH_MAX ];
};

__device__ __forceinline__ unsigned udiv_q1( unsigned n, const udiv_t & v )
{
    return v.d == 1 ? n : udiv_q( n, v );
}

// Item it of work list `list`: x group, y block, z plane, w tile.  Uniform over
// the CTA when it is (it comes from blockIdx and the loop counter).
template< class R > __device__ __forceinline__
int4 batch_item( const multi_t< R > & m, int list, int it )
{
    int p = 0;
#pragma unroll
    for( int q = 1; q < KR_BATCH_MAX; ++ q )
        if( q < m.ng && it >= m.l_off[ list ][ q ] )
            p = q;
    const unsigned r = unsigned( it - m.l_off[ list ][ p ] );
    const udiv_t & dt = m.l_tiles[ list ][ p ], & dp = m.l_planes[ list ][ p ];
    const unsigned q = udiv_q1( r, dt );              // block * planes + plane
    const unsigned b = udiv_q1( q, dp );
    return make_int4( m.l_grp[ list ][ p ], int( b ), int( q - b * dp.d ), int( r - q * dt.d ) );
}

struct multi_scal_t
{
    scal_t * s[ KR_BATCH_MAX ];
    int ns[ KR_BATCH_MAX ];
    int n;
};

__global__ void k_step_begin_multi( const __grid_constant__ multi_scal_t m )
{
    for( int g = 0; g < m.n; ++ g )
        for( int k = 0; k < m.ns[ g ]; ++ k )
            m.s[ g ][ k ].dt_bits = __double_as_longlong( m.s[ g ][ k ].dt_bound );
}

__global__ void k_step_end_multi( const __grid_constant__ multi_scal_t m, double dt_expand )
{
    for( int g = 0; g < m.n; ++ g )
        for( int k = 0; k < m.ns[ g ]; ++ k )
        {
            scal_t & r = m.s[ g ][ k ];
            const double dt = __longlong_as_double( r.dt_bits );
            if( ! ( dt > 0 ) || ! isfinite( dt ) )
                m.s[ g ][ 0 ].status |= 1;
            r.dt_last  = dt;
            r.t       += dt;
            r.dt_bound = dt * dt_expand;
            r.n_steps += 1;
            r.sel_force = 0;
        }
}

// item: x group, y block, z plane, w tile
template< bool MHD, class R, bool DT >
__global__ void __launch_bounds__( 256, ( MHD && DT ) ? 3 : 4 )
k_c2p_list( const __grid_constant__ multi_t< R > m, int step, int n_items )
{
    for( int it = blockIdx.x; it < n_items; it += gridDim.x )
    {
        const int4 t = batch_item( m, 0, it );
        c2p_cells< MHD, R, DT >( m.a[ t.x ], step, m.dv_c[ t.x ], t.y, t.z, unsigned( t.w ) * 256u + threadIdx.x );
        if( DT )
            __syncthreads(  );            // the CTA reduction's shared words are reused
    }
}

// MODE: the step's solver; KR_RIEMANN_LEARNED launches the network's sweep
// (stage 0 of an evaluation step only), FLUX_APPLY the other sweeps.
// AXIS is a template argument: with a runtime axis, the per-group arguments
// read through the item's group index left an 80-byte local array in the
// kernel (the per-size k_flux has none).
template< bool MHD, class R, int MODE, int AXIS >
__global__ void __launch_bounds__( 128, ( flux_min_ctas< R, MODE >(  ) ) )
k_flux_list( const __grid_constant__ multi_t< R > m, int step, int n_items )
{
    constexpr int axis = AXIS;
    if constexpr( MODE == KR_RIEMANN_LEARNED || MODE == FLUX_APPLY )
    {   // every group steps in lockstep: group 0's scalars decide
        const bool eval = step == 0 && sel_eval_step( m.a[ 0 ].s, m.a[ 0 ].sel_period );
        if( eval != ( MODE == KR_RIEMANN_LEARNED ) )
            return;
    }
    for( int it = blockIdx.x; it < n_items; it += gridDim.x )
    {
        const int4 t = batch_item( m, 1 + ( 2 - axis ), it );
        const args_t< R > & a = m.a[ t.x ];
        if constexpr( MODE == FLUX_APPLY )
        {
            const bool hlle = ( a.sel_dec[ ( ( size_t ) axis * a.nblk + t.y ) * a.sel_wcap
                                           + ( unsigned( t.z ) * m.cpp_f[ axis ][ t.x ] + unsigned( t.w ) ) * 4u
                                           + ( threadIdx.x >> 5 ) ] >> ( threadIdx.x & 31 ) ) & 1u;
            flux_faces< MHD, R, FLUX_APPLY >( a, axis, step, m.dv_f[ axis ][ t.x ], t.y, t.w, t.z, hlle );
        }
        else
            flux_faces< MHD, R, MODE >( a, axis, step, m.dv_f[ axis ][ t.x ], t.y, t.w, t.z );
    }
}

template< class R >
__global__ void __launch_bounds__( 256 )
k_emf_list( const __grid_constant__ multi_t< R > m, int n_items )
{
    for( int it = blockIdx.x; it < n_items; it += gridDim.x )
    {
        const int4 t = batch_item( m, 4, it );
        emf_site< R >( m.a[ t.x ], m.dv_e[ t.x ], t.y, t.z, unsigned( t.w ) * 256u + threadIdx.x );
    }
}

template< bool MHD, class R, int PART >
__global__ void __launch_bounds__( 256, ( PART == 2 ? 6 : 4 ) )
k_update_list( const __grid_constant__ multi_t< R > m, int step, int n_items )
{
    for( int it = blockIdx.x; it < n_items; it += gridDim.x )
    {
        const int4 t = batch_item( m, 4, it );
        update_site< MHD, R, false, PART >( m.a[ t.x ], step, m.dv_e[ t.x ], t.y, t.z, unsigned( t.w ) * 256u + threadIdx.x );
    }
}

// Stage 0's update, CT and stage 1's c2p in one launch (update_c2p_cell), over
// the c2p work list (item: x group, y block, z plane, w tile of 256 cells).
template< class R >
__global__ void __launch_bounds__( 256, 3 )
k_update_c2p_list( const __grid_constant__ multi_t< R > m, int n_items )
{
    for( int it = blockIdx.x; it < n_items; it += gridDim.x )
    {
        const int4 t = batch_item( m, 0, it );
        const args_t< R > & a = m.a[ t.x ];
        const unsigned c = unsigned( t.w ) * 256u + threadIdx.x;
        if( c >= unsigned( a.n0 * a.n1 ) )
            continue;
        const unsigned q = udiv_q( c, m.dv_c[ t.x ] );
        update_c2p_cell< R >( a, t.y, int( c - q * unsigned( a.n0 ) ), int( q ), t.z );
    }
}

// Launch kinds with a tunable grid, in this order in kr_batch::grid.
enum { BK_C2P0, BK_C2P1, BK_FLUX, BK_EVAL, BK_EMF, BK_UPD1, BK_UPD2, BK_UPDC2P, BK_N };
static const char * const BK_NAME[ BK_N ] = { "c2p0", "c2p1", "flux", "eval", "emf", "upd1", "upd2", "updc2p" };
// resident CTAs per SM each kind is compiled for (its __launch_bounds__)
template< class R > static int bk_min_ctas( int k )
{
    switch( k )
    {
    case BK_C2P0: return 3;
    case BK_C2P1: return 4;
    case BK_FLUX: return flux_min_ctas< R, FLUX_APPLY >(  );
    case BK_EVAL: return flux_min_ctas< R, KR_RIEMANN_LEARNED >(  );
    case BK_EMF:  return 4;
    case BK_UPD1: return 4;
    case BK_UPDC2P: return 3;
    default:      return 6;
    }
}
}   // namespace kr

struct kr_batch
{
    std::vector< kr_ctx * > ctx;
    std::string err;
    int precision = 2, riemann = 0;
    // work lists: [c2p | flux z | flux y | flux x | lattice sites], ordered
    // bigger blocks first (decoded on the device, batch_item)
    long long cnt[ 5 ] = { 0 };
    int l_off[ 5 ][ KR_BATCH_MAX + 1 ] = { { 0 } }, l_grp[ 5 ][ KR_BATCH_MAX ] = { { 0 } };
    kr::udiv_t l_tiles[ 5 ][ KR_BATCH_MAX ] = { }, l_planes[ 5 ][ KR_BATCH_MAX ] = { };
    bool fuse = false;                   // every context fuses stage 0's update with stage 1's c2p
    int grid[ kr::BK_N ] = { 0 };        // CTAs per launch kind (0: one per item)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector< float > thr;            // selector thresholds the graph was built with
    int n_sm = 148;
    cudaEvent_t ev = nullptr;            // orders the contexts' streams around a step
};

namespace kr
{
static bool bck( kr_batch * b, cudaError_t e, const char * what )
{
    if( e == cudaSuccess ) return true;
    b->err = std::string( what ) + ": " + cudaGetErrorString( e );
    return false;
}

template< class R >
static multi_t< R > make_multi( kr_batch * bt )
{
    multi_t< R > m;
    std::memset( ( void * ) & m, 0, sizeof( m ) );
    for( size_t g = 0; g < bt->ctx.size(  ); ++ g )
    {
        kr_ctx * c = bt->ctx[ g ];
        const int * n = c->cfg.n;
        m.a[ g ] = make_args< R >( c );
        m.dv_c[ g ] = make_udiv( unsigned( n[ 0 ] ) );
        m.dv_e[ g ] = make_udiv( unsigned( n[ 0 ] + 1 ) );
        for( int axis = 0; axis < 3; ++ axis )
        {
            int ext[ 3 ];
            for( int d = 0; d < 3; ++ d )
                ext[ d ] = ( d == axis ) ? n[ d ] + 1 : n[ d ] + 2;
            m.dv_f[ axis ][ g ] = make_udiv( unsigned( ext[ 0 ] ) );
            m.cpp_f[ axis ][ g ] = unsigned( blocks_for( ( long long ) ext[ 0 ] * ext[ 1 ], 128 ) );
        }
    }
    m.ng = int( bt->ctx.size(  ) );
    std::memcpy( m.l_off, bt->l_off, sizeof( m.l_off ) );
    std::memcpy( m.l_grp, bt->l_grp, sizeof( m.l_grp ) );
    std::memcpy( m.l_tiles, bt->l_tiles, sizeof( m.l_tiles ) );
    std::memcpy( m.l_planes, bt->l_planes, sizeof( m.l_planes ) );
    return m;
}

static multi_scal_t make_multi_scal( kr_batch * bt )
{
    multi_scal_t m;
    std::memset( ( void * ) & m, 0, sizeof( m ) );
    m.n = int( bt->ctx.size(  ) );
    for( int g = 0; g < m.n; ++ g )
    {
        m.s[ g ] = bt->ctx[ g ]->s;
        m.ns[ g ] = bt->ctx[ g ]->nscal;
    }
    return m;
}

static unsigned bgrid( const kr_batch * bt, int kind, int list )
{
    const long long n = bt->cnt[ list ];
    const long long g = bt->grid[ kind ] > 0 ? std::min< long long >( bt->grid[ kind ], n ) : n;
    return unsigned( std::max< long long >( 1, g ) );
}

// One Heun step of every group; `timed` wraps each launch (kind index).
template< class R, class T >
static void batch_enqueue( kr_batch * bt, cudaStream_t st, T && timed )
{
    const multi_t< R > m = make_multi< R >( bt );
    const multi_scal_t ms = make_multi_scal( bt );
    k_step_begin_multi<<< 1, 1, 0, st >>>( ms );
    const bool learned = bt->riemann == KR_RIEMANN_LEARNED;
    for( int stage = 0; stage < 2; ++ stage )
    {
        if( ! ( bt->fuse && stage == 1 ) )        // (fused: stage 0's update did stage 1's c2p)
            timed( stage ? BK_C2P1 : BK_C2P0, [ & ] {
                ( stage == 0 ? k_c2p_list< true, R, true > : k_c2p_list< true, R, false > )
                    <<< bgrid( bt, stage ? BK_C2P1 : BK_C2P0, 0 ), 256, 0, st >>>( m, stage, int( bt->cnt[ 0 ] ) ); } );
        for( int axis = 2; axis >= 0; -- axis )
        {
            const int list = 1 + ( 2 - axis );
            const int nl = int( bt->cnt[ list ] );
            auto sweep = [ & ]( int kind, auto mode )
            {
                constexpr int M = decltype( mode )::value;
                const unsigned g = bgrid( bt, kind, list );
                timed( kind, [ & ] {
                    if( axis == 0 )      k_flux_list< true, R, M, 0 ><<< g, 128, 0, st >>>( m, stage, nl );
                    else if( axis == 1 ) k_flux_list< true, R, M, 1 ><<< g, 128, 0, st >>>( m, stage, nl );
                    else                 k_flux_list< true, R, M, 2 ><<< g, 128, 0, st >>>( m, stage, nl ); } );
            };
            if( learned )
            {
                sweep( BK_EVAL, std::integral_constant< int, KR_RIEMANN_LEARNED >(  ) );
                sweep( BK_FLUX, std::integral_constant< int, FLUX_APPLY >(  ) );
            }
            else if( bt->riemann == KR_RIEMANN_HLLE )
                sweep( BK_FLUX, std::integral_constant< int, KR_RIEMANN_HLLE >(  ) );
            else
                sweep( BK_FLUX, std::integral_constant< int, KR_RIEMANN_DEFAULT >(  ) );
        }
        const int ne = int( bt->cnt[ 4 ] );
        timed( BK_EMF, [ & ] { k_emf_list< R ><<< bgrid( bt, BK_EMF, 4 ), 256, 0, st >>>( m, ne ); } );
        if( bt->fuse && stage == 0 )
        {
            timed( BK_UPDC2P, [ & ] {
                k_update_c2p_list< R ><<< bgrid( bt, BK_UPDC2P, 0 ), 256, 0, st >>>( m, int( bt->cnt[ 0 ] ) ); } );
            continue;
        }
        timed( BK_UPD1, [ & ] { k_update_list< true, R, 1 ><<< bgrid( bt, BK_UPD1, 4 ), 256, 0, st >>>( m, stage, ne ); } );
        timed( BK_UPD2, [ & ] { k_update_list< true, R, 2 ><<< bgrid( bt, BK_UPD2, 4 ), 256, 0, st >>>( m, stage, ne ); } );
    }
    k_step_end_multi<<< 1, 1, 0, st >>>( ms, bt->ctx[ 0 ]->cfg.dt_expand );
}

static void batch_drop_graph( kr_batch * bt )
{
    if( bt->exec ) cudaGraphExecDestroy( bt->exec );
    if( bt->graph ) cudaGraphDestroy( bt->graph );
    bt->exec = nullptr;
    bt->graph = nullptr;
}

static bool batch_build_graph( kr_batch * bt )
{
    batch_drop_graph( bt );
    cudaStream_t st = bt->ctx[ 0 ]->stream;
    if( ! bck( bt, cudaStreamBeginCapture( st, cudaStreamCaptureModeThreadLocal ), "capture begin" ) )
        return false;
    if( bt->precision == 1 ) batch_enqueue< float >( bt, st, untimed_t(  ) );
    else                     batch_enqueue< double >( bt, st, untimed_t(  ) );
    const bool ended = bck( bt, cudaStreamEndCapture( st, & bt->graph ), "capture end" );
    if( ! ended || ! bck( bt, cudaGraphInstantiate( & bt->exec, bt->graph, 0 ), "graph instantiate" ) )
    {
        const std::string e = bt->err;
        batch_drop_graph( bt );
        bt->err = e;
        return false;
    }
    bt->thr.clear(  );
    for( kr_ctx * c : bt->ctx )
        bt->thr.push_back( c->sel_thr );
    return true;
}

// One eager step with CUDA events around every launch: ms[kind] summed.
static bool batch_profile_step( kr_batch * bt, double * ms )
{
    cudaStream_t st = bt->ctx[ 0 ]->stream;
    cudaEvent_t ev[ 2 ];
    cudaEventCreate( & ev[ 0 ] );
    cudaEventCreate( & ev[ 1 ] );
    auto timed = [ & ]( int kind, auto && launch )
    {
        cudaEventRecord( ev[ 0 ], st );
        launch(  );
        cudaEventRecord( ev[ 1 ], st );
        cudaEventSynchronize( ev[ 1 ] );
        float t = 0;
        cudaEventElapsedTime( & t, ev[ 0 ], ev[ 1 ] );
        ms[ kind ] += t;
    };
    if( bt->precision == 1 ) batch_enqueue< float >( bt, st, timed );
    else                     batch_enqueue< double >( bt, st, timed );
    cudaEventDestroy( ev[ 0 ] );
    cudaEventDestroy( ev[ 1 ] );
    return bck( bt, cudaStreamSynchronize( st ), "batch profile" );
}

// The state a tuning step changes: both RK slots of U and BF (the step reads
// slot 1 only after writing it, but the pushed ghost strips live in both), the
// scalars and the selector's decisions and counters.
struct batch_saved_t
{
    std::vector< std::vector< std::pair< void *, void * > > > bufs;   // (live, copy)
    std::vector< std::vector< size_t > > bytes;
};

static bool batch_save( kr_batch * bt, batch_saved_t & sv, bool restore )
{
    if( ! restore )
    {
        sv.bufs.assign( bt->ctx.size(  ), { } );
        sv.bytes.assign( bt->ctx.size(  ), { } );
    }
    for( size_t g = 0; g < bt->ctx.size(  ); ++ g )
    {
        kr_ctx * c = bt->ctx[ g ];
        if( ! restore )
        {
            auto add = [ & ]( void * p, size_t n )
            {
                if( ! p || ! n ) return true;
                void * q = nullptr;
                if( ! bck( bt, cudaMalloc( & q, n ), "autotune: save buffer" ) )
                    return false;
                sv.bufs[ g ].push_back( { p, q } );
                sv.bytes[ g ].push_back( n );
                return true;
            };
            const size_t nu = size_t( c->nblk ) * 5 * c->nc * sizeof( double );
            const size_t nb = size_t( c->nblk ) * 3 * c->nbf * sizeof( double );
            if( ! add( c->u[ 0 ], nu ) || ! add( c->u[ 1 ], nu ) || ! add( c->bf[ 0 ], nb ) || ! add( c->bf[ 1 ], nb )
                || ! add( c->s, size_t( c->nscal ) * sizeof( scal_t ) )
                || ! add( c->sel_cnt, c->sel_cnt ? 2 * sizeof( unsigned long long ) : 0 )
                || ! add( c->sel_dec, c->sel_dec ? size_t( 3 ) * c->nblk * c->sel_wcap * sizeof( unsigned ) : 0 ) )
                return false;
        }
        for( size_t k = 0; k < sv.bufs[ g ].size(  ); ++ k )
        {
            void * live = sv.bufs[ g ][ k ].first, * copy = sv.bufs[ g ][ k ].second;
            if( ! bck( bt, cudaMemcpyAsync( restore ? live : copy, restore ? copy : live, sv.bytes[ g ][ k ],
                                            cudaMemcpyDeviceToDevice, bt->ctx[ 0 ]->stream ), "autotune: copy state" ) )
                return false;
        }
    }
    return bck( bt, cudaStreamSynchronize( bt->ctx[ 0 ]->stream ), "autotune: sync" );
}

static void batch_free_saved( batch_saved_t & sv )
{
    for( auto & v : sv.bufs )
        for( auto & p : v )
            cudaFree( p.second );
    sv.bufs.clear(  );
}

static std::string batch_key( const kr_batch * bt )
{
    cudaDeviceProp prop;
    cudaGetDeviceProperties( & prop, bt->ctx[ 0 ]->cfg.device );
    std::string k = "kr_batch v2 ";
    for( const char * p = prop.name; * p; ++ p )
        k += ( * p == ' ' ) ? '_' : * p;
    k += " sm" + std::to_string( prop.multiProcessorCount ) + " prec" + std::to_string( bt->precision )
       + " riemann" + std::to_string( bt->riemann );
    for( kr_ctx * c : bt->ctx )
        k += " " + std::to_string( c->cfg.n[ 0 ] ) + "x" + std::to_string( c->nblk );
    return k;
}
}   // namespace kr

extern "C" {

kr_batch * kr_batch_create( kr_ctx * const * ctxs, int n )
{
    using namespace kr;
    g_create_error.clear(  );
    if( ! ctxs || n < 1 || n > KR_BATCH_MAX )
    {
        g_create_error = "kr_batch_create: need 1.." + std::to_string( KR_BATCH_MAX ) + " contexts";
        return nullptr;
    }
    for( int g = 0; g < n; ++ g )
    {
        const kr_ctx * c = ctxs[ g ];
        if( ! c || ! c->boxes || ! c->cfg.mhd )
        {
            g_create_error = "kr_batch_create: every context must be a KR_FLAG_BOXES (MHD) context";
            return nullptr;
        }
        if( c->cfg.device != ctxs[ 0 ]->cfg.device || c->cfg.precision != ctxs[ 0 ]->cfg.precision
            || c->cfg.riemann != ctxs[ 0 ]->cfg.riemann || c->cfg.dt_expand != ctxs[ 0 ]->cfg.dt_expand
            || c->cfg.sel_period != ctxs[ 0 ]->cfg.sel_period )
        {
            g_create_error = "kr_batch_create: the contexts differ in device, precision, solver, dt_expand or sel_period";
            return nullptr;
        }
    }
    kr_batch * bt = new kr_batch;
    bt->ctx.assign( ctxs, ctxs + n );
    bt->precision = ctxs[ 0 ]->cfg.precision;
    bt->riemann = ctxs[ 0 ]->cfg.riemann;
    bt->n_sm = ctxs[ 0 ]->n_sm;
    cudaSetDevice( ctxs[ 0 ]->cfg.device );
    // the uniform launches' CTA tiles, bigger blocks first
    std::vector< int > order( n );
    for( int g = 0; g < n; ++ g ) order[ g ] = g;
    std::stable_sort( order.begin(  ), order.end(  ), [ & ]( int x, int y ) { return ctxs[ x ]->cfg.n[ 0 ] > ctxs[ y ]->cfg.n[ 0 ]; } );
    bt->fuse = true;
    for( int g = 0; g < n; ++ g )
        bt->fuse = bt->fuse && ctxs[ g ]->fuse_batch;
    for( int list = 0; list < 5; ++ list )
    {
        long long count = 0;
        for( int p = 0; p < n; ++ p )
        {
            const int g = order[ p ];
            const int * nn = ctxs[ g ]->cfg.n;
            long long tiles, planes;
            if( list == 0 )      { tiles = blocks_for( ( long long ) nn[ 0 ] * nn[ 1 ], 256 ); planes = nn[ 2 ]; }
            else if( list == 4 ) { tiles = blocks_for( ( long long )( nn[ 0 ] + 1 ) * ( nn[ 1 ] + 1 ), 256 ); planes = nn[ 2 ] + 1; }
            else
            {
                const int axis = 2 - ( list - 1 );
                int ext[ 3 ];
                for( int d = 0; d < 3; ++ d )
                    ext[ d ] = ( d == axis ) ? nn[ d ] + 1 : nn[ d ] + 2;
                tiles = blocks_for( ( long long ) ext[ 0 ] * ext[ 1 ], 128 );
                planes = ext[ 2 ];
            }
            bt->l_off[ list ][ p ] = int( count );
            bt->l_grp[ list ][ p ] = g;
            bt->l_tiles[ list ][ p ] = make_udiv( unsigned( tiles ) );
            bt->l_planes[ list ][ p ] = make_udiv( unsigned( planes ) );
            const long long items = tiles * planes * ctxs[ g ]->nblk;
            // the multiply-high quotients are exact while item * divisor < 2^32
            if( items * std::max( tiles, planes ) >= ( 1LL << 32 ) )
            {
                g_create_error = "kr_batch_create: a box group's work list is too long for 32-bit item decoding";
                delete bt;
                return nullptr;
            }
            count += items;
        }
        if( count >= ( 1LL << 31 ) )
        {
            g_create_error = "kr_batch_create: a work list of more than 2^31 items";
            delete bt;
            return nullptr;
        }
        bt->l_off[ list ][ n ] = int( count );
        bt->cnt[ list ] = count;
    }
    for( int k = 0; k < BK_N; ++ k )          // default: 4 waves of resident CTAs
        bt->grid[ k ] = 4 * bt->n_sm * ( bt->precision == 1 ? bk_min_ctas< float >( k ) : bk_min_ctas< double >( k ) );
    return bt;
}

void kr_batch_destroy( kr_batch * bt )
{
    if( ! bt ) return;
    cudaSetDevice( bt->ctx[ 0 ]->cfg.device );
    kr::batch_drop_graph( bt );
    if( bt->ev ) cudaEventDestroy( bt->ev );
    delete bt;
}

const char * kr_batch_last_error( const kr_batch * bt )
{
    return bt ? bt->err.c_str(  ) : g_create_error.c_str(  );
}

int kr_batch_step( kr_batch * bt, int n_steps )
{
    using namespace kr;
    if( ! bt || n_steps < 0 ) return -1;
    for( kr_ctx * c : bt->ctx )
        if( bt->riemann == KR_RIEMANN_LEARNED && ! c->sel_ready )
        {
            bt->err = "kr_batch_step: learned face selector configured but no weights set (kr_set_selector)";
            return -1;
        }
    cudaSetDevice( bt->ctx[ 0 ]->cfg.device );
    bool stale = ! bt->exec || bt->thr.size(  ) != bt->ctx.size(  );
    for( size_t g = 0; ! stale && g < bt->ctx.size(  ); ++ g )
        stale = bt->thr[ g ] != bt->ctx[ g ]->sel_thr;
    if( stale && ! batch_build_graph( bt ) )
        return -1;
    // the steps run on the first context's stream: after the work already
    // enqueued on every context's stream, and before whatever comes next there
    cudaStream_t s0 = bt->ctx[ 0 ]->stream;
    if( ! bt->ev && ! bck( bt, cudaEventCreateWithFlags( & bt->ev, cudaEventDisableTiming ), "batch event" ) )
        return -1;
    for( size_t g = 1; g < bt->ctx.size(  ); ++ g )
        if( ! bck( bt, cudaEventRecord( bt->ev, bt->ctx[ g ]->stream ), "batch event" )
            || ! bck( bt, cudaStreamWaitEvent( s0, bt->ev, 0 ), "batch wait" ) )
            return -1;
    for( int s = 0; s < n_steps; ++ s )
        if( ! bck( bt, cudaGraphLaunch( bt->exec, s0 ), "batch graph launch" ) )
            return -1;
    if( ! bck( bt, cudaEventRecord( bt->ev, s0 ), "batch event" ) )
        return -1;
    for( size_t g = 1; g < bt->ctx.size(  ); ++ g )
        if( ! bck( bt, cudaStreamWaitEvent( bt->ctx[ g ]->stream, bt->ev, 0 ), "batch wait" ) )
            return -1;
    return 0;
}

int kr_batch_launches_per_step( kr_batch * bt )
{
    if( ! bt ) return -1;
    const int flux = bt->riemann == KR_RIEMANN_LEARNED ? 6 : 3;
    // fused: stage 0's two updates and stage 1's c2p are one launch
    return 2 + 2 * ( 1 + flux + 3 ) - ( bt->fuse ? 2 : 0 );
}

int kr_batch_profile_step( kr_batch * bt, int n_kinds, double * ms )
{
    using namespace kr;
    if( ! bt || ! ms || n_kinds < BK_N ) return -1;
    for( kr_ctx * c : bt->ctx )
        if( bt->riemann == KR_RIEMANN_LEARNED && ! c->sel_ready )
        {
            bt->err = "kr_batch_profile_step: learned face selector configured but no weights set";
            return -1;
        }
    cudaSetDevice( bt->ctx[ 0 ]->cfg.device );
    for( int k = 0; k < BK_N; ++ k ) ms[ k ] = 0;
    return batch_profile_step( bt, ms ) ? 0 : -1;
}

int kr_batch_get_grid( kr_batch * bt, int * grid )
{
    if( ! bt || ! grid ) return -1;
    for( int k = 0; k < kr::BK_N; ++ k )
        grid[ k ] = bt->grid[ k ];
    return kr::BK_N;
}

int kr_batch_set_grid( kr_batch * bt, const int * grid )
{
    if( ! bt || ! grid ) return -1;
    for( int k = 0; k < kr::BK_N; ++ k )
        if( grid[ k ] < 0 )
        {
            bt->err = "kr_batch_set_grid: negative CTA count";
            return -1;
        }
    for( int k = 0; k < kr::BK_N; ++ k )
        bt->grid[ k ] = grid[ k ];
    kr::batch_drop_graph( bt );
    return 0;
}

int kr_batch_autotune( kr_batch * bt, const char * cache_path, int * grid_out )
{
    using namespace kr;
    if( ! bt ) return -1;
    cudaSetDevice( bt->ctx[ 0 ]->cfg.device );
    const std::string key = batch_key( bt );
    if( cache_path && * cache_path )
    {   // a line "<key> | c2p0=.. c2p1=.. ..." from an earlier tuning
        FILE * f = std::fopen( cache_path, "r" );
        if( f )
        {
            char line[ 4096 ];
            bool hit = false;
            while( ! hit && std::fgets( line, sizeof( line ), f ) )
            {
                const std::string l( line );
                const size_t bar = l.find( " | " );
                if( bar == std::string::npos || l.compare( 0, bar, key ) != 0 || bar != key.size(  ) )
                    continue;
                int g[ BK_N ];
                int got = 0;
                for( int k = 0; k < BK_N; ++ k )
                {
                    const std::string tag = std::string( " " ) + BK_NAME[ k ] + "=";
                    const size_t p = l.find( tag, bar );
                    if( p != std::string::npos )
                    {
                        g[ k ] = std::atoi( l.c_str(  ) + p + tag.size(  ) );
                        ++ got;
                    }
                }
                if( got == BK_N )
                {
                    for( int k = 0; k < BK_N; ++ k ) bt->grid[ k ] = g[ k ];
                    hit = true;
                }
            }
            std::fclose( f );
            if( hit )
            {
                batch_drop_graph( bt );
                if( grid_out ) kr_batch_get_grid( bt, grid_out );
                return 1;
            }
        }
    }
    // Candidates per launch kind: 1, 2, 4 and 8 waves of resident CTAs, and one
    // CTA per work item.  Each candidate set is timed over two eager steps on a
    // copy of the state (restored afterwards), and every kind keeps its fastest.
    batch_saved_t sv;
    if( ! batch_save( bt, sv, false ) )
    {
        batch_free_saved( sv );
        return -1;
    }
    const int waves[ ] = { 1, 2, 4, 8, 0 };
    double best[ BK_N ];
    int pick[ BK_N ];
    for( int k = 0; k < BK_N; ++ k ) { best[ k ] = 1e300; pick[ k ] = bt->grid[ k ]; }
    bool ok = true;
    for( int w : waves )
    {
        for( int k = 0; k < BK_N; ++ k )
            bt->grid[ k ] = w ? w * bt->n_sm * ( bt->precision == 1 ? bk_min_ctas< float >( k ) : bk_min_ctas< double >( k ) ) : 0;
        double ms[ BK_N ] = { 0 };
        for( int rep = 0; rep < 3 && ok; ++ rep )
        {
            double once[ BK_N ] = { 0 };
            ok = batch_profile_step( bt, once );
            if( rep > 0 )                     // the first step warms up
                for( int k = 0; k < BK_N; ++ k ) ms[ k ] += once[ k ];
        }
        ok = ok && batch_save( bt, sv, true );
        if( ! ok ) break;
        for( int k = 0; k < BK_N; ++ k )
            if( ms[ k ] < best[ k ] )
            {
                best[ k ] = ms[ k ];
                pick[ k ] = bt->grid[ k ];
            }
    }
    batch_free_saved( sv );
    for( int k = 0; k < BK_N; ++ k ) bt->grid[ k ] = pick[ k ];
    batch_drop_graph( bt );
    if( ! ok ) return -1;
    if( cache_path && * cache_path )
    {
        FILE * f = std::fopen( cache_path, "a" );
        if( f )
        {
            std::fprintf( f, "%s |", key.c_str(  ) );
            for( int k = 0; k < BK_N; ++ k )
                std::fprintf( f, " %s=%d", BK_NAME[ k ], bt->grid[ k ] );
            std::fprintf( f, "\n" );
            std::fclose( f );
        }
    }
    if( grid_out ) kr_batch_get_grid( bt, grid_out );
    return 0;
}

}   // extern "C"
