// Drop-in adapter: the reference solver with its hot-path tasks on the GPU.
// (The incompressible solver's UPDATE_RESIDUALS likewise, in its own task
// table system/ins/function/funcMap.txt: OfgInsUpdateResiduals below.)
//
// Linked into a second build of the reference (oneflow_ref_ofg, see the
// Makefile beside this file) whose task tables system/{ns,turb}/function/
// funcMap.txt map the task names of TimeIntegral::Lusgs
// (codes/solver/src/TimeIntegral.cpp:113-130) -- ZERO_DQ_FIELD,
// CALC_TIME_STEP, LOAD_RESIDUALS, UPDATE_RESIDUALS, INIT_LUSGS,
// LUSGS_LOWER_SWEEP, LUSGS_UPPER_SWEEP, UPDATE_FLOWFIELD_LUSGS, CALC_BOUNDARY
// -- to the classes registered here instead of the reference's own
// (CNsCalcTimeStep, CNsUpdateResiduals, CLusgsLowerSweep, ...).  Every other
// task (initialisation, restart, residual and force output, visualisation)
// stays the reference's.  The reference dispatches a task by name
// (SsSgTask, codes/task/src/CmxTask.cpp:152-159) to HXClone::Solve() of the
// class its table names; the classes below call the C ABI of
// oneflow_b200/libofg.so with the solver of SolverState::tid.
//
// Data flow: the first task of a solve creates the GPU context from the
// reference's own zone (nodes, face->node lists, lCells/rCells, boundary
// codes, wall distance), its script keys and its initialised fields (q,
// turbq).  From then on the state lives on the GPU; after each task the
// fields that the reference's remaining tasks read are copied back into its
// host fields: the residual and the gradients after UPDATE_RESIDUALS (the
// residual output and the force integration read them; the boundary-face
// gradients are filled as Grad::StoreBcGrad does, codes/grad/src/Grad.cpp:131-156),
// the state with its ghost cells, temperature and viscosities after
// CALC_BOUNDARY.  Test infrastructure: it shows the boundary working from the
// reference's side; the product path is the C ABI itself.
#include "CellMesh.h"
#include "DataBase.h"
#include "FaceTopo.h"
#include "BcRecord.h"
#include "HXClone.h"
#include "Iteration.h"
#include "NodeMesh.h"
#include "SolverDef.h"
#include "SolverState.h"
#include "UnsGrid.h"
#include "Zone.h"
#include "BcData.h"
#include "INsBcSolver.h"
#include "INsInvterm.h"
#include "INsIdx.h"
#include "HXMath.h"

#include <cstdio>
#include <iostream>
#include <cstdlib>
#include <string>
#include <vector>

#include "oneflow_b200.h"

BeginNameSpace( ONEFLOW )

namespace {

ofg_ctx *g_ctx = nullptr;
ofg_ins *g_ins = nullptr;
bool g_turb = false;

void Check( int rc, const char *what )
{
    if ( rc == OFG_OK ) return;
    std::fprintf( stderr, "oneflow_b200: %s failed (%d): %s\n", what, rc, ofg_last_error( g_ctx ) );
    std::exit( 3 );
}

// the C ABI's solver of the reference's SolverState::tid (NS_SOLVER = 1,
// TURB_SOLVER = 2, codes/global/include/SolverDef.h:31-32)
int Tid()
{
    return SolverState::tid == TURB_SOLVER ? OFG_TURB_SOLVER : OFG_NS_SOLVER;
}

template < typename T >
T Key( const std::string & name, T fallback )
{
    DataBase * db = ONEFLOW::GetGlobalDataBase();
    return db->dataPara->GetDataPointer( name ) ? ONEFLOW::GetDataValue< T >( name, db ) : fallback;
}

// The reference's script keys on this path -> ofg_params (the struct's
// fields carry the same names).
void ReadParams( ofg_params & p )
{
    ofg_default_params( & p );
    p.dimension = Key< int >( "dimension", p.dimension );
    p.ischeme = Key< int >( "ischeme", p.ischeme );
    p.ilim = Key< int >( "ilim", p.ilim );
    p.ieigenfix = Key< int >( "ieigenfix", p.ieigenfix );
    p.timestepModel = Key< int >( "timestepModel", p.timestepModel );
    p.ncfl = Key< int >( "ncfl", p.ncfl );
    p.visSRModel = Key< int >( "visSRModel", p.visSRModel );
    p.visTimeStepModel = Key< int >( "visTimeStepModel", p.visTimeStepModel );
    p.vismodel = Key< int >( "vismodel", p.vismodel );
    p.ivischeme = Key< int >( "ivischeme", p.ivischeme );
    p.isowallbc = Key< int >( "isowallbc", p.isowallbc );
    p.iprod_sa = Key< int >( "iprod_sa", p.iprod_sa );
    p.ft2_flag = Key< int >( "ft2_flag", p.ft2_flag );
    p.turb_ilim = Key< int >( "turb_ilim", p.turb_ilim );
    p.time_integral = Key< int >( "time_integral", p.time_integral );
    // 3 (SIMPLE) is the incompressible solver's integrator, which has its own
    // entry points; the context underneath it keeps the LU-SGS default
    if ( p.time_integral == 3 ) p.time_integral = 2;
    p.vencat_coef = Key< Real >( "vencat_coef", p.vencat_coef );
    p.centropy1 = Key< Real >( "centropy1", p.centropy1 );
    p.centropy2 = Key< Real >( "centropy2", p.centropy2 );
    p.cflst = Key< Real >( "cflst", p.cflst );
    p.cfled = Key< Real >( "cfled", p.cfled );
    p.max_time_ratio = Key< Real >( "max_time_ratio", p.max_time_ratio );
    p.global_dt = Key< Real >( "global_dt", p.global_dt );
    p.mach_ref = Key< Real >( "mach_ref", p.mach_ref );
    p.aoa_degree = Key< Real >( "aoa_degree", p.aoa_degree );
    p.sideslip_degree = Key< Real >( "sideslip_degree", p.sideslip_degree );
    p.reynolds = Key< Real >( "reynolds", p.reynolds );
    p.gama_ref = Key< Real >( "gama_ref", p.gama_ref );
    p.prl = Key< Real >( "prl", p.prl );
    p.prt = Key< Real >( "prt", p.prt );
    p.tref_dim = Key< Real >( "tref_dim", p.tref_dim );
    p.twall_dim = Key< Real >( "twall_dim", p.twall_dim );
    p.inflow_viscosity = Key< Real >( "inflow_viscosity", p.inflow_viscosity );
    p.rprod = Key< Real >( "rprod", p.rprod );
    p.turb_cfl_ratio = Key< Real >( "turb_cfl_ratio", p.turb_cfl_ratio );
    p.ref_sa = Key< Real >( "ref_sa", p.ref_sa );
    p.max_vis_ratio = Key< Real >( "max_vis_ratio", p.max_vis_ratio );
    // the reference's own arithmetic and sweep order: the FP64 path
    p.precision = OFG_PREC_FP64;
    p.sweep_order = 0;
}

void Flatten( MRField & f, std::vector< double > & out )
{
    int ne = f.GetNEqu(), n = f[ 0 ].size();
    out.resize( (size_t)ne * n );
    for ( int e = 0; e < ne; ++ e )
        for ( int i = 0; i < n; ++ i ) out[ (size_t)e * n + i ] = f[ e ][ i ];
}

void Unflatten( const std::vector< double > & in, MRField & f )
{
    int ne = f.GetNEqu(), n = f[ 0 ].size();
    for ( int e = 0; e < ne; ++ e )
        for ( int i = 0; i < n; ++ i ) f[ e ][ i ] = in[ (size_t)e * n + i ];
}

// GPU field -> the reference's host field of the same name and layout
void Download( UnsGrid * grid, int tid, const char * name, const char * hostName )
{
    MRField * f = GetFieldPointer< MRField >( grid, hostName );
    std::vector< double > buf( (size_t)f->GetNEqu() * ( * f )[ 0 ].size() );
    int64_t need = 0;
    Check( ofg_download_field( g_ctx, tid, name, buf.data(), (int64_t)buf.size(), & need ), name );
    if ( need != (int64_t)buf.size() )
    {
        std::fprintf( stderr, "oneflow_b200: field %s has %lld values, host field %s %zu\n", name, (long long)need,
                      hostName, buf.size() );
        std::exit( 3 );
    }
    Unflatten( buf, * f );
}

// the context and the zone's mesh (nodes, face->node lists, lCells/rCells,
// boundary codes, SA wall distance)
void CreateMeshContext()
{
    UnsGrid * grid = Zone::GetUnsGrid();
    ofg_params p;
    ReadParams( p );
    Check( ofg_create( & p, & g_ctx ), "ofg_create" );
    FaceTopo * ft = grid->faceTopo;
    // the boundary-face count lives in the BC record (FaceTopo::GetNBFaces)
    int nFaces = ft->faces.size(), nCells = grid->nCells, nBFaces = (int)ft->GetNBFaces();
    std::vector< int > fnc( nFaces ), fn, lc( nFaces ), rc( nFaces );
    for ( int f = 0; f < nFaces; ++ f )
    {
        fnc[ f ] = ft->faces[ f ].size();
        for ( int v : ft->faces[ f ] ) fn.push_back( v );
        lc[ f ] = ft->lCells[ f ];
        rc[ f ] = f < nBFaces ? -1 : ft->rCells[ f ];
    }
    IntField & bct = ft->bcManager->bcRecord->bcType;
    std::vector< int > bc( bct.begin(), bct.begin() + nBFaces );
    NodeMesh * nm = grid->nodeMesh;
    g_turb = p.vismodel >= 3;
    RealField & dist = grid->cellMesh->dist;
    const double * wd = ( g_turb && (int)dist.size() >= nCells ) ? dist.data() : nullptr;
    Check( ofg_upload_mesh( g_ctx, nm->xN.size(), nm->xN.data(), nm->yN.data(), nm->zN.data(), nFaces, fnc.data(),
                            fn.data(), lc.data(), rc.data(), nCells, nBFaces, bc.data(), wd ), "ofg_upload_mesh" );
}

void CreateContext()
{
    CreateMeshContext();
    UnsGrid * grid = Zone::GetUnsGrid();
    int nCells = grid->nCells, nFaces = grid->faceTopo->faces.size();
    std::vector< double > buf;
    Flatten( * GetFieldPointer< MRField >( grid, "q" ), buf );
    Check( ofg_upload_state( g_ctx, OFG_NS_SOLVER, buf.data() ), "ofg_upload_state (NS)" );
    if ( g_turb )
    {
        Flatten( * GetFieldPointer< MRField >( grid, "turbq" ), buf );
        Check( ofg_upload_state( g_ctx, OFG_TURB_SOLVER, buf.data() ), "ofg_upload_state (SA)" );
    }
    std::fprintf( stderr, "oneflow_b200: hot-path tasks on the GPU (%d cells, %d faces%s)\n", nCells, nFaces,
                  g_turb ? ", NS + SA" : "" );
}

}  // namespace

// ZERO_DQ_FIELD: the first task of every outer iteration of each solver; the
// NS one also carries the reference's outer-step counter (the CFL ramp)
void OfgZeroDq( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    if ( Tid() == OFG_NS_SOLVER ) Check( ofg_set_outer_step( g_ctx, Iteration::outerSteps ), "ofg_set_outer_step" );
    Check( ofg_zero_dq( g_ctx, Tid() ), "ofg_zero_dq" );
}

// (every task creates the context if it is the first one to run)
void OfgCalcTimeStep( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_calc_time_step( g_ctx, Tid() ), "ofg_calc_time_step" );
}

void OfgLoadResiduals( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_load_residuals( g_ctx, Tid() ), "ofg_load_residuals" );
}

void OfgInitLusgs( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_init_lusgs( g_ctx, Tid() ), "ofg_init_lusgs" );
}

void OfgLowerSweep( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_lusgs_lower( g_ctx, Tid() ), "ofg_lusgs_lower" );
}

void OfgUpperSweep( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_lusgs_upper( g_ctx, Tid() ), "ofg_lusgs_upper" );
}

void OfgUpdateFlowField( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    Check( ofg_update_flowfield( g_ctx, Tid() ), "ofg_update_flowfield" );
}

void OfgUpdateResiduals( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    int tid = Tid();
    Check( ofg_update_residuals( g_ctx, tid ), "ofg_update_residuals" );
    UnsGrid * grid = Zone::GetUnsGrid();
    if ( tid == OFG_TURB_SOLVER )
    {
        Download( grid, tid, "turbres", "turbres" );
        return;
    }
    Download( grid, tid, "res", "res" );
    const char * g[ 3 ] = { "dqdx", "dqdy", "dqdz" };
    const char * bg[ 3 ] = { "bcdqdx", "bcdqdy", "bcdqdz" };
    FaceTopo * ft = grid->faceTopo;
    for ( int d = 0; d < 3; ++ d )
    {
        // ghost cells carry their interior cell's gradient (UGrad.cpp:140-148),
        // boundary faces that of their interior cell (Grad::StoreBcGrad)
        Download( grid, tid, g[ d ], g[ d ] );
        MRField & cell = * GetFieldPointer< MRField >( grid, g[ d ] );
        MRField & bc = * GetFieldPointer< MRField >( grid, bg[ d ] );
        for ( int f = 0; f < (int)ft->GetNBFaces(); ++ f )
        {
            int lc = ft->lCells[ f ];
            for ( int e = 0; e < (int)cell.GetNEqu(); ++ e ) cell[ e ][ grid->nCells + f ] = cell[ e ][ lc ];
            for ( int e = 0; e < (int)bc.GetNEqu(); ++ e ) bc[ e ][ f ] = cell[ e ][ lc ];
        }
    }
}

void OfgCalcBoundary( StringField & data )
{
    if ( ! g_ctx ) CreateContext();
    int tid = Tid();
    Check( ofg_calc_boundary( g_ctx, tid ), "ofg_calc_boundary" );
    UnsGrid * grid = Zone::GetUnsGrid();
    if ( tid == OFG_TURB_SOLVER )
    {
        MRField * tq = GetFieldPointer< MRField >( grid, "turbq" );
        std::vector< double > buf( ( * tq )[ 0 ].size() );
        Check( ofg_download_state( g_ctx, tid, buf.data() ), "ofg_download_state (SA)" );
        Unflatten( buf, * tq );
        Download( grid, OFG_NS_SOLVER, "vist", "vist" );
        return;
    }
    MRField * q = GetFieldPointer< MRField >( grid, "q" );
    std::vector< double > buf( (size_t)q->GetNEqu() * ( * q )[ 0 ].size() );
    Check( ofg_download_state( g_ctx, tid, buf.data() ), "ofg_download_state (NS)" );
    Unflatten( buf, * q );
    Download( grid, tid, "tempr", "tempr" );
    Download( grid, tid, "visl", "visl" );
}

// UPDATE_RESIDUALS of the incompressible solver (system/ins/function/
// funcMap.txt; CINsUpdateResiduals -> INsCalcRHS, codes/ins/src/INsRhs.cpp:105-132):
// one inner SIMPLE iteration on the GPU.  The first call builds the solver
// from the zone, the wall velocities of the ins_bc data (per boundary face,
// through its bcNameId region, as UINsBcSolver::SetId reads them,
// codes/uins/src/UINsBcSolver.cpp:64-81) and the state INIT_FINAL left in q.
// Afterwards q and the gradients go back to the host fields, and the residual
// maxima to iinv, whose remax_up/vp/wp MG::Run's inner loop tests
// (codes/multigrid/src/Multigrid.cpp:132-141); they are printed as
// UINsInvterm::UpdateINsRes prints them.
void OfgInsUpdateResiduals( StringField & data )
{
    UnsGrid * grid = Zone::GetUnsGrid();
    MRField * q = GetFieldPointer< MRField >( grid, "q" );
    std::vector< double > buf;
    if ( ! g_ins )
    {
        CreateMeshContext();
        FaceTopo * ft = grid->faceTopo;
        int nBFaces = (int)ft->GetNBFaces();
        IntField & bcn = ft->bcManager->bcRecord->bcNameId;
        std::vector< double > wall( 3 * (size_t)nBFaces, 0.0 );
        for ( int f = 0; f < nBFaces; ++ f )
        {
            int id = bcn[ f ];
            if ( id < 0 || id >= (int)ins_bc_data.r2d.size() ) continue;
            int dd = ins_bc_data.r2d[ id ];
            if ( dd == -1 ) continue;
            for ( int k = 0; k < 3; ++ k ) wall[ 3 * f + k ] = ins_bc_data.dataList[ dd ][ IIDX::IIU + k ];
        }
        Check( ofg_ins_create( g_ctx, wall.data(), & g_ins ), "ofg_ins_create" );
        Flatten( * q, buf );
        Check( ofg_ins_upload_state( g_ins, buf.data() ), "ofg_ins_upload_state" );
        std::fprintf( stderr, "oneflow_b200: incompressible inner iterations on the GPU (%d cells)\n", grid->nCells );
    }
    Check( ofg_ins_update_residuals( g_ins ), "ofg_ins_update_residuals" );
    buf.resize( (size_t)q->GetNEqu() * ( * q )[ 0 ].size() );
    Check( ofg_ins_get_field( g_ins, "q", buf.data(), (int64_t)buf.size() ), "ofg_ins_get_field q" );
    Unflatten( buf, * q );
    const char * g[ 3 ] = { "dqdx", "dqdy", "dqdz" };
    for ( int d = 0; d < 3; ++ d )
    {
        MRField * f = GetFieldPointer< MRField >( grid, g[ d ] );
        Check( ofg_ins_get_field( g_ins, g[ d ], buf.data(), (int64_t)buf.size() ), g[ d ] );
        Unflatten( buf, * f );
    }
    double st[ 13 ];
    Check( ofg_ins_stats( g_ins, st ), "ofg_ins_stats" );
    iinv.remax_up = st[ 0 ];
    iinv.remax_vp = st[ 1 ];
    iinv.remax_wp = st[ 2 ];
    iinv.remax_pp = st[ 3 ];
    std::cout << "iinv.remax_up:" << iinv.remax_up << std::endl;
    std::cout << "iinv.remax_vp:" << iinv.remax_vp << std::endl;
    std::cout << "iinv.remax_wp:" << iinv.remax_wp << std::endl;
    std::cout << "iinv.remax_pp:" << iinv.remax_pp << std::endl;
}

DEFINE_DATA_CLASS( OfgZeroDq );
DEFINE_DATA_CLASS( OfgCalcTimeStep );
DEFINE_DATA_CLASS( OfgLoadResiduals );
DEFINE_DATA_CLASS( OfgUpdateResiduals );
DEFINE_DATA_CLASS( OfgInitLusgs );
DEFINE_DATA_CLASS( OfgLowerSweep );
DEFINE_DATA_CLASS( OfgUpperSweep );
DEFINE_DATA_CLASS( OfgUpdateFlowField );
DEFINE_DATA_CLASS( OfgCalcBoundary );
DEFINE_DATA_CLASS( OfgInsUpdateResiduals );

namespace {
// registered at load time (HXClone::Register keeps a lazily created map)
struct OfgRegistrar
{
    OfgRegistrar()
    {
        REGISTER_DATA_CLASS( OfgZeroDq );
        REGISTER_DATA_CLASS( OfgCalcTimeStep );
        REGISTER_DATA_CLASS( OfgLoadResiduals );
        REGISTER_DATA_CLASS( OfgUpdateResiduals );
        REGISTER_DATA_CLASS( OfgInitLusgs );
        REGISTER_DATA_CLASS( OfgLowerSweep );
        REGISTER_DATA_CLASS( OfgUpperSweep );
        REGISTER_DATA_CLASS( OfgUpdateFlowField );
        REGISTER_DATA_CLASS( OfgCalcBoundary );
        REGISTER_DATA_CLASS( OfgInsUpdateResiduals );
    }
} g_registrar;
}  // namespace

EndNameSpace
