/* CPU restatement (FP64) of the Kratos unsplit Godunov hydro / ideal-MHD step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA implementation of
 * the package is checked against; nothing in the product links or calls it.
 *
 * Scope: a Cartesian mesh of nb[0] x nb[1] x nb[2] root blocks, optionally
 * statically refined (restriction / prolongation of the ghost cells across a
 * level jump and the flux correction of the coarse side; MHD also the face-B
 * restriction, Toth-Roe face-B prolongation and the edge-E correction, on
 * periodic domains), two ghost layers (PLM), Heun RK2 (two stages per step).
 *   hydro : adiabatic EOS, PLM (van Leer harmonic limiter), HLLC.
 *   mhd   : adiabatic EOS with face-centred B, PLM, HLLD, Gardiner-Stone
 *           upwinded edge EMF (constrained transport), CT face update.
 * Every function cites the reference file:line it restates (paths relative to
 * the Kratos source tree).  The arithmetic follows the reference expression by
 * expression, so a build without fused multiply-add reproduces the reference's
 * own CPU build bit for bit.
 *
 * Storage (one array per block, AoS with the field index fastest, x fastest
 * among cells, as mesh/types/dat_3d.h:153-156):
 *   u  : n0*n1*n2 cells x nw            (nw = 5 hydro, 8 MHD), no ghosts
 *   bf : (n0+5)(n1+5)(n2+5) x 3         face field on the (n+1)^3 lattice with
 *                                       2 ghost layers, as the snapshot stores it
 * Blocks are numbered level by level, lexicographically (x fastest) inside a
 * level; a uniform mesh is one level.
 */
#ifndef KR_ORACLE_H
#define KR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { KRO_PER = 0, KRO_OUT = 1, KRO_REF = 2, KRO_FRE = 3, KRO_FIXD = 4 };

typedef struct
{
    int    mhd;              /* 0: hydro (PLM + HLLC), 1: MHD (PLM + HLLD + CT) */
    int    nb[ 3 ];          /* blocks per axis                                 */
    int    n [ 3 ];          /* cells per block per axis (all > 1)              */
    double x_min[ 3 ], x_max[ 3 ];
    double gamma, cfl, d_floor, t_floor;
    double dt_expand;        /* [cycle] dt_expand                               */
    int    n_threads;        /* host threads used (<= 0: all)                   */
    /* [boundary] kinds per side (x-, x+, y-, y+, z-, z+): KRO_PER, KRO_OUT,
     * KRO_REF, KRO_FRE, KRO_FIXD (hydro/boundary/phys_functors.h); an axis is
     * periodic only if both its sides are KRO_PER. */
    int    bc[ 6 ];
    double w_fix[ 5 ];       /* [init] rho0, pre0, vel0 for KRO_FIXD            */
    double b_fix[ 3 ];       /* [init] b0 for KRO_FIXD (MHD)                    */
    int    integrator;       /* 0: Heun RK2 (the reference's rk2_t); 1: VL2     */
} kro_cfg;

typedef struct kro_mesh kro_mesh;

/* A static refinement region ([refine_region*] section: level, x_min, x_max). */
typedef struct
{
    int    level;
    double x_min[ 3 ], x_max[ 3 ];
} kro_region;

kro_mesh * kro_create ( const kro_cfg * cfg );
/* A mesh with static refinement: the leaves of the block tree
 * that the regions build (meshgen.cpp:111-160, tree.cpp:139-232), numbered
 * level by level, lexicographically inside a level.  With no region (or only
 * level-0 regions) this is kro_create's uniform mesh.  NULL for a region
 * outside the domain.  kro_step returns -2 on a refined MHD mesh with a
 * non-periodic axis (physical sides across a level jump are not restated). */
kro_mesh * kro_create_tree( const kro_cfg * cfg, int n_regions, const kro_region * regions );
int        kro_nblk   ( const kro_mesh * m );
/* Level and logical position (at that level) of every block: level[nblk],
 * reg[nblk][3]. */
void       kro_block_info( const kro_mesh * m, int * level, int * reg );
void       kro_destroy( kro_mesh * m );
int        kro_nw     ( const kro_mesh * m );
long       kro_ncell  ( const kro_mesh * m );   /* cells per block          */
long       kro_nface  ( const kro_mesh * m );   /* bf lattice sites / block */

/* Copy the slot-0 state in / out (all blocks, layouts above). */
void kro_set_state( kro_mesh * m, const double * u, const double * bf );
void kro_get_state( const kro_mesh * m, double * u, double * bf );

/* Advance n_steps Heun steps.  *dt_bound is the device dt value a step starts
 * from (cycle.cpp:77-115: the CFL minimum is taken against it; afterwards it is
 * dt_use * dt_expand).  Returns the dt of the last step through *dt_last and
 * advances *t.  Returns 0, or -1 on a non-finite dt. */
/* cons -> prim (floors heal slot 0) and each block's CFL dt of slot 0. */
void kro_c2p_dt( kro_mesh * m, double * w_out, double * dt_out );
int  kro_step( kro_mesh * m, int n_steps, double * t, double * dt_bound,
               double * dt_last );

/* Block geometry as meshgen computes it (meshgen.cpp:252-363): cell-centre and
 * face coordinates along an axis, and the cell size of a block. */
double kro_x_cc( const kro_mesh * m, int block, int axis, int i );
double kro_x_fc( const kro_mesh * m, int block, int axis, int i );
double kro_dx  ( const kro_mesh * m, int block, int axis );

/* Seeded initial state of a named workload ("shock" or "ot"), built from the
 * shared initial-condition header (kratos_b200/csrc/problems.h) with this
 * mesh's geometry, into slot 0.  Returns 0, or -1 for an unknown name. */
int kro_init_problem( kro_mesh * m, const char * name, unsigned long long seed );
/* box `box` of a batch of independent periodic MHD boxes (problems.h kr_box_*) */
int kro_init_box( kro_mesh * m, unsigned long long seed, int box );
int kro_box_n( unsigned long long seed, int box );

/* Single-face kernels, for unit tests of the restatement.  Inputs are primitive
 * left / right states (rho, p, v0, v1, v2 [, b0, b1, b2]) in the unrotated
 * frame; the flux comes back in the unrotated frame (HLLD: with the B flux
 * already remapped to the edge EMF, hlld.h:35-47). */
void kro_hllc( const double * ql, const double * qr, int axis, double gamma,
               double * flx );
void kro_hlld( const double * ql, const double * qr, int axis, double gamma,
               double * flx );
void kro_plm ( const double * q4, double * ql, double * qr );

#ifdef __cplusplus
}
#endif
#endif
