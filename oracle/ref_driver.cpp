// Oracle build of the reference itself (test infrastructure only).
//
// Compiles the reference's own Sparse::CholeskyDecomposition headers, read in
// place from the reference checkout, against the project-written stand-in for
// their missing utility submodule (oracle/shim) and scipy's bundled OpenBLAS,
// and exposes a small C interface so that tests and the CPU-baseline leg of
// bench.py can drive the unmodified reference code path:
//   constructor (CholeskyDecomposition.hpp:313-345), SymbolicFactorization
//   (CholeskyDecomposition/Symbolic.hpp:3), NumericFactorization
//   (CholeskyDecomposition/Numeric.hpp:3), Solve / LowerSolve
//   (CholeskyDecomposition/Solve.hpp:22,248), getters
//   (CholeskyDecomposition/InputOutput.hpp:259-367).
// UpperSolve (Solve.hpp:182) is not exposed: it declares its tag as a
// constexpr std::string built from run-time arguments (Solve.hpp:188), so it
// cannot be instantiated by a conforming compiler.
// The library is built by oracle/Makefile into oracle/_ref/libtb_ref.so.

#include "submodules/Tools/Tools.hpp"

namespace Tensors { using namespace Tools; }

#include "src/Tensor1.hpp"
#include "src/Tensor2.hpp"

#include <cblas.h>
#include <lapack.h>

namespace Tensors
{
    namespace BLAS
    {
        using Int           = blasint;
        using Bool          = bool;
        using ComplexFloat  = lapack_complex_float;
        using ComplexDouble = lapack_complex_double;
    }
    namespace LAPACK
    {
        using Int           = lapack_int;
        using Bool          = bool;
        using ComplexFloat  = lapack_complex_float;
        using ComplexDouble = lapack_complex_double;
    }
}

#include "src/BLAS_Wrappers.hpp"
#include "src/LAPACK_Wrappers.hpp"

#include "src/Sorting/TwoArraySort.hpp"
#include "src/Sorting/ThreeArraySort.hpp"
#include "src/Aggregator.hpp"
#include "src/PairAggregator.hpp"
#include "src/TripleAggregator.hpp"
#include "src/AssemblyCounters.hpp"
#include "src/Sparse/Permutation.hpp"
namespace Tensors {
    // PatternCSR names these in members that the Cholesky path never instantiates.
    template<typename Scal, IntQ Int, IntQ LInt> class SparseBLAS;
    namespace Tiny { template<int n_, typename Scal_, IntQ Int_, Size_T alignment = DefaultAlignment> class VectorList_AoS; }
}
#include "src/Sparse/PatternCSR.hpp"
#include "src/Sparse/BinaryMatrixCSR.hpp"

// MatrixCSR carries the MatrixMarket reader and writer (MatrixCSR/MatrixMarket.hpp).
#include "src/Sparse/MatrixCSR.hpp"

#include "Sparse.hpp"

#include <cstdint>
#include <memory>

using namespace Tensors;

namespace
{
    using Int  = std::int32_t;
    using LInt = std::int64_t;
    using Chol = Sparse::CholeskyDecomposition<double, Int, LInt, Parallel>;
    using Mat  = Sparse::MatrixCSR<double, Int, LInt, Parallel>;

    struct RefHandle
    {
        std::unique_ptr<Chol> chol;
        Int threads = 1;
    };

    template<typename T>
    void copy_out( const T * src, std::int64_t n, std::int64_t * dst )
    {
        for( std::int64_t i = 0; i < n; ++i ) { dst[i] = static_cast<std::int64_t>(src[i]); }
    }
}

extern "C"
{

void tb_ref_set_quiet( int quiet ) { Tools::LogQuiet() = (quiet != 0); }

void tb_ref_set_blas_threads( int t ) { scipy_openblas_set_num_threads( t ); }

// perm may be null: then the matrix is taken as already permuted
// (CholeskyDecomposition.hpp:350); otherwise perm[i] is the original index
// placed at position i (CholeskyDecomposition.hpp:336, Inverse::False).
void * tb_ref_create( int n, const std::int64_t * outer, const std::int32_t * inner,
                      const std::int32_t * perm, int threads )
{
    auto * h = new RefHandle();
    h->threads = threads < 1 ? 1 : threads;
    if( perm != nullptr )
    {
        h->chol = std::make_unique<Chol>( outer, inner, perm, Int(n), Int(h->threads) );
    }
    else
    {
        h->chol = std::make_unique<Chol>( outer, inner, Int(n), Int(h->threads) );
    }
    return h;
}

void tb_ref_destroy( void * p ) { delete static_cast<RefHandle*>(p); }

void tb_ref_set_strategy( void * p, int s )
{
    static_cast<RefHandle*>(p)->chol->SetSupernodeStrategy( static_cast<Chol::SupernodeStrategy_T>(s) );
}

void tb_ref_set_amalgamation_threshold( void * p, int t )
{
    static_cast<RefHandle*>(p)->chol->SetAmalgamationThreshold( Int(t) );
}

void tb_ref_set_method( void * p, int m )
{
    static_cast<RefHandle*>(p)->chol->SetFactorizationMethod( static_cast<Chol::FactorizationMethod_T>(m) );
}

void tb_ref_symbolic( void * p ) { static_cast<RefHandle*>(p)->chol->SymbolicFactorization(); }

int tb_ref_sn_count( void * p ) { return static_cast<RefHandle*>(p)->chol->SN_Count(); }

// Array selectors: 0 perm, 1 inverse perm, 2 value permutation, 3 SN_rp,
// 4 SN_outer, 5 SN_inner, 6 row_to_SN, 7 SN_tri_ptr, 8 SN_rec_ptr,
// 9 assembly-tree parents, 10 elimination-tree parents, 11 permuted outer,
// 12 permuted inner, 13 assembly-tree child pointers, 14 child indices.
std::int64_t tb_ref_array_size( void * p, int which )
{
    auto & c = *static_cast<RefHandle*>(p)->chol;
    switch( which )
    {
        case 0:  return c.GetPermutation().GetPermutation().Size();
        case 1:  return c.GetPermutation().GetInversePermutation().Size();
        case 2:  return c.GetValuePermutation().Size();
        case 3:  return c.SN_RowPointers().Size();
        case 4:  return c.SN_Outer().Size();
        case 5:  return c.SN_Inner().Size();
        case 6:  return c.RowToSN().Size();
        case 7:  return c.SN_TrianglePointers().Size();
        case 8:  return c.SN_RectanglePointers().Size();
        case 9:  return c.AssemblyTree().Parents().Size();
        case 10: return c.EliminationTree().Parents().Size();
        case 11: return c.GetA().Outer().Size();
        case 12: return c.GetA().Inner().Size();
        case 13: return c.AssemblyTree().ChildPointers().Size();
        case 14: return c.AssemblyTree().ChildIndices().Size();
        default: return -1;
    }
}

void tb_ref_array_copy( void * p, int which, std::int64_t * out )
{
    auto & c = *static_cast<RefHandle*>(p)->chol;
    const std::int64_t n = tb_ref_array_size( p, which );
    switch( which )
    {
        case 0:  copy_out( c.GetPermutation().GetPermutation().data(), n, out ); break;
        case 1:  copy_out( c.GetPermutation().GetInversePermutation().data(), n, out ); break;
        case 2:  copy_out( c.GetValuePermutation().data(), n, out ); break;
        case 3:  copy_out( c.SN_RowPointers().data(), n, out ); break;
        case 4:  copy_out( c.SN_Outer().data(), n, out ); break;
        case 5:  copy_out( c.SN_Inner().data(), n, out ); break;
        case 6:  copy_out( c.RowToSN().data(), n, out ); break;
        case 7:  copy_out( c.SN_TrianglePointers().data(), n, out ); break;
        case 8:  copy_out( c.SN_RectanglePointers().data(), n, out ); break;
        case 9:  copy_out( c.AssemblyTree().Parents().data(), n, out ); break;
        case 10: copy_out( c.EliminationTree().Parents().data(), n, out ); break;
        case 11: copy_out( c.GetA().Outer().data(), n, out ); break;
        case 12: copy_out( c.GetA().Inner().data(), n, out ); break;
        case 13: copy_out( c.AssemblyTree().ChildPointers().data(), n, out ); break;
        case 14: copy_out( c.AssemblyTree().ChildIndices().data(), n, out ); break;
        default: break;
    }
}

int tb_ref_numeric( void * p, const double * values, double reg )
{
    return static_cast<RefHandle*>(p)->chol->NumericFactorization( values, reg );
}

int tb_ref_good( void * p ) { return static_cast<RefHandle*>(p)->chol->NumericallyGoodQ() ? 1 : 0; }

std::int64_t tb_ref_tri_size( void * p ) { return static_cast<RefHandle*>(p)->chol->SN_TriangleValues().Size(); }
std::int64_t tb_ref_rec_size( void * p ) { return static_cast<RefHandle*>(p)->chol->SN_RectangleValues().Size(); }

void tb_ref_tri_copy( void * p, double * out )
{
    const auto & v = static_cast<RefHandle*>(p)->chol->SN_TriangleValues();
    copy_buffer( v.data(), out, static_cast<Size_T>(v.Size()) );
}

void tb_ref_rec_copy( void * p, double * out )
{
    const auto & v = static_cast<RefHandle*>(p)->chol->SN_RectangleValues();
    copy_buffer( v.data(), out, static_cast<Size_T>(v.Size()) );
}

// X = alpha * A^{-1} B + beta * X with row-major n x nrhs blocks.
void tb_ref_solve( void * p, double alpha, const double * B, int ldB,
                   double beta, double * X, int ldX, int nrhs, int parallel )
{
    auto & c = *static_cast<RefHandle*>(p)->chol;
    if( parallel )
    {
        c.Solve<VarSize,Parallel>( alpha, B, Int(ldB), beta, X, Int(ldX), Int(nrhs) );
    }
    else
    {
        c.Solve<VarSize,Sequential>( alpha, B, Int(ldB), beta, X, Int(ldX), Int(nrhs) );
    }
}

void tb_ref_lower_solve( void * p, double alpha, const double * B, int ldB,
                         double beta, double * X, int ldX, int nrhs )
{
    static_cast<RefHandle*>(p)->chol->LowerSolve<VarSize,Sequential>( alpha, B, Int(ldB), beta, X, Int(ldX), Int(nrhs) );
}

double tb_ref_log_det( void * p ) { return static_cast<RefHandle*>(p)->chol->LogDeterminant(); }

void tb_ref_factor_diagonal( void * p, double * diag ) { static_cast<RefHandle*>(p)->chol->WriteFactorDiagonal( diag ); }

// MatrixMarket files through Sparse::MatrixCSR::LoadFromMatrixMarket
// (MatrixCSR/MatrixMarket.hpp:3-202).  A file the reference rejects leaves the
// matrix empty (0 x 0).  Its WriteToMatrixMarket is not bound: its merge step
// (MatrixMarket.hpp:296-305) appends thread_strings[2 * thread + 2] for
// thread 1, one past its four slices, and never writes slices 1 and 3.
void * tb_ref_mm_load( const char * path, int threads )
{
    auto * A = new Mat();
    A->LoadFromMatrixMarket( std::filesystem::path( path ), Int( threads < 1 ? 1 : threads ) );
    return A;
}

void tb_ref_mm_sizes( void * p, std::int32_t * rows, std::int32_t * cols, std::int64_t * nnz )
{
    auto & A = *static_cast<Mat*>(p);
    *rows = A.RowCount(); *cols = A.ColCount(); *nnz = A.NonzeroCount();
}

void tb_ref_mm_copy( void * p, std::int64_t * outer, std::int32_t * inner, double * values )
{
    auto & A = *static_cast<Mat*>(p);
    if( A.RowCount() <= 0 ) { return; }
    for( Int i = 0; i <= A.RowCount(); ++i ) { outer[i] = A.Outer()[i]; }
    for( LInt k = 0; k < A.NonzeroCount(); ++k ) { inner[k] = A.Inner()[k]; values[k] = A.Values()[k]; }
}

void tb_ref_mm_free( void * p ) { delete static_cast<Mat*>(p); }

} // extern "C"
