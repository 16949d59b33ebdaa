// tensors_b200::Sparse::CholeskyDecomposition -- header-only C++ mirror of
// Tensors::Sparse::CholeskyDecomposition<Scal,Int,LInt,parQ>
// (src/Sparse/CholeskyDecomposition.hpp) over the C-ABI of tensors_b200.h.
//
// Member names, argument order and argument meaning follow the reference so
// that code written against it compiles after swapping the include and the
// namespace.  Template arguments: Scal = double (FP64 factor) or float (FP32
// factor storage with 3xTF32 tensor-core updates; solves are refined in FP64
// to the handle's target, so they are at least as accurate as the reference's
// float solves); Int = int32_t and LInt = int64_t, as the reference's driver
// instantiates it (Example_SparseCholesky/main.cpp:31-32).  The reference's
// parQ argument selects host threading and has no counterpart: every
// numeric phase runs on the GPU.  Differences:
//  - errors throw tensors_b200::Sparse::Error (the reference prints with
//    eprint and continues); NumericFactorization still returns 1 for a
//    non-positive pivot, like the reference (Numeric.hpp:99);
//  - LowerSolve solves with U^T as documented (the reference's LowerSolve
//    runs the upper solve, Solve.hpp:290-307);
//  - the template arguments of the reference's Solve (NRHS, parQ, op) are not
//    needed: the right-hand-side count is a run-time argument and every solve
//    runs on the GPU; the scalar types of B and X are the call's own (float
//    or double, cast on copy as Solve.hpp:20-27).
// Link with tensors_b200/libtensors_b200.so (the library built by
// tensors_b200/build.py).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../tensors_b200.h"
#include "Error.hpp"
#include "MatrixCSR.hpp"

namespace tensors_b200 {
namespace Sparse {

enum class SupernodeStrategy_T : int32_t
{
    Maximal = TB_SN_MAXIMAL, Fundamental = TB_SN_FUNDAMENTAL, Amalgamated = TB_SN_AMALGAMATED
};

enum class FactorizationMethod_T : int32_t
{
    Multifrontal = TB_MULTIFRONTAL, LeftLooking = TB_LEFT_LOOKING
};

namespace detail
{
template<typename T> constexpr int32_t dtype_of()
{
    static_assert( std::is_same<T, double>::value || std::is_same<T, float>::value, "scalars are double or float" );
    return std::is_same<T, float>::value ? TB_F32 : TB_F64;
}
} // namespace detail

template<typename Scal_ = double, typename Int_ = int32_t, typename LInt_ = int64_t>
class CholeskyDecomposition
{
public:
    using Scal = Scal_;
    using Int  = Int_;
    using LInt = LInt_;
    static_assert( std::is_same<Scal, double>::value || std::is_same<Scal, float>::value, "Scal is double or float" );
    static_assert( std::is_same<Int, int32_t>::value && std::is_same<LInt, int64_t>::value,
                   "Int = int32_t and LInt = int64_t (the reference driver's instantiation)" );

    // NumericalFactorization_T (CholeskyDecomposition.hpp:132-201): a numeric
    // factor held apart from any decomposition, exchanged by
    // SwapNumericalFactorization.  Device memory; a new one is empty.
    class NumericalFactorization_T
    {
    public:
        NumericalFactorization_T() { Check( tb_factor_create( &f_ ) ); }
        ~NumericalFactorization_T() { if( f_ != nullptr ) { tb_factor_destroy( f_ ); } }
        NumericalFactorization_T( const NumericalFactorization_T & ) = delete;
        NumericalFactorization_T & operator=( const NumericalFactorization_T & ) = delete;
        NumericalFactorization_T( NumericalFactorization_T && o ) noexcept : f_( std::exchange( o.f_, nullptr ) ) {}

        bool NumericallyFactorizedQ() const { int32_t f = 0; Check( tb_factor_state( f_, &f, nullptr, nullptr, nullptr ) ); return f != 0; }
        bool NumericallyGoodQ() const { int32_t g = 0; Check( tb_factor_state( f_, nullptr, &g, nullptr, nullptr ) ); return g != 0; }
        size_t AllocatedByteCount() const { int64_t b = 0; Check( tb_factor_state( f_, nullptr, nullptr, &b, nullptr ) ); return static_cast<size_t>( b ); }
        tb_factor * Handle() const noexcept { return f_; }

    private:
        tb_factor * f_ = nullptr;
    };

    // Fill-reducing permutation p of size n (Inverse::False), ctor
    // CholeskyDecomposition.hpp:336-346.  thread_count is used by the host
    // symbolic phase.
    CholeskyDecomposition( const LInt * A_outer, const Int * A_inner, const Int * p,
                           Int n, Int thread_count )
    : threads_( thread_count )
    {
        Check( tb_chol_create( &h_, n, A_outer, A_inner, p, thread_count ) );
        SetScalarPrecision();
    }

    // Matrix already permuted, ctor CholeskyDecomposition.hpp:350-371.
    CholeskyDecomposition( const LInt * A_outer, const Int * A_inner, Int n, Int thread_count )
    : threads_( thread_count )
    {
        Check( tb_chol_create( &h_, n, A_outer, A_inner, nullptr, thread_count ) );
        SetScalarPrecision();
    }

    ~CholeskyDecomposition() { if( h_ != nullptr ) { tb_chol_destroy( h_ ); } }

    CholeskyDecomposition( const CholeskyDecomposition & ) = delete;
    CholeskyDecomposition & operator=( const CholeskyDecomposition & ) = delete;
    CholeskyDecomposition( CholeskyDecomposition && o ) noexcept
    :   h_( std::exchange( o.h_, nullptr ) ), strategy_( o.strategy_ ), threshold_( o.threshold_ ), method_( o.method_ ),
        threads_( o.threads_ ), cg_iter_( o.cg_iter_ ), restarts_( o.restarts_ ), relres_( std::move( o.relres_ ) ) {}
    CholeskyDecomposition & operator=( CholeskyDecomposition && o ) noexcept
    {
        if( this != &o )
        {
            if( h_ != nullptr ) { tb_chol_destroy( h_ ); }
            h_ = std::exchange( o.h_, nullptr );
            strategy_ = o.strategy_; threshold_ = o.threshold_; method_ = o.method_; threads_ = o.threads_;
            cg_iter_ = o.cg_iter_; restarts_ = o.restarts_; relres_ = std::move( o.relres_ );
        }
        return *this;
    }

    // Setters, CholeskyDecomposition/InputOutput.hpp:369-409.
    void SetSupernodeStrategy( SupernodeStrategy_T s )
    {
        Check( tb_chol_set_supernode_strategy( h_, static_cast<int32_t>( s ) ) );
        strategy_ = s;
    }
    void SetAmalgamationThreshold( Int t ) { Check( tb_chol_set_amalgamation_threshold( h_, t ) ); threshold_ = t; }
    void SetFactorizationMethod( FactorizationMethod_T m )
    {
        Check( tb_chol_set_factorization_method( h_, static_cast<int32_t>( m ) ) );
        method_ = m;
    }
    // The settings' getters (InputOutput.hpp) and the thread count given to the constructor.
    SupernodeStrategy_T GetSupernodeStrategy() const { return strategy_; }
    Int AmalgamationThreshold() const { return threshold_; }
    FactorizationMethod_T GetFactorizationMethod() const { return method_; }
    Int ThreadCount() const { return threads_; }

    // CholeskyDecomposition/Symbolic.hpp:3-66.
    void SymbolicFactorization() { Check( tb_chol_symbolic( h_ ) ); }

    // CholeskyDecomposition/Numeric.hpp:3-24: values in the caller's CSR
    // order, reg added to the diagonal.  0 = success, 1 = not positive
    // definite.  ExtScal is the values' own type (float or double), cast on
    // copy as NumericFactorization<ExtScal> does.
    template<typename ExtScal>
    int NumericFactorization( const ExtScal * A_val, ExtScal reg = ExtScal( 0 ) )
    {
        return Check( tb_chol_numeric_ex( h_, A_val, detail::dtype_of<ExtScal>(), static_cast<double>( reg ) ) );
    }
    // Same with A_val in device memory of the handle's GPU.
    template<typename ExtScal>
    int NumericFactorization_Device( const ExtScal * d_A_val, ExtScal reg = ExtScal( 0 ) )
    {
        return Check( tb_chol_numeric_device_ex( h_, d_A_val, detail::dtype_of<ExtScal>(), static_cast<double>( reg ) ) );
    }

    // SwapNumericalFactorization (Numeric.hpp:228-254): exchanges this
    // object's numeric factor with cont.  A factor that says factorized but
    // not good, or is smaller than this symbolic analysis requires, is then
    // treated as unfactorized.
    void SwapNumericalFactorization( NumericalFactorization_T & cont ) { Check( tb_chol_swap_factor( h_, cont.Handle() ) ); }

    // X_out = alpha * A^{-1} B + beta * X_out, row-major n x nrhs
    // (Solve.hpp:22-80); host pointers.  B and X_out each float or double.
    template<typename B_T, typename X_T>
    void Solve( double alpha, const B_T * B, Int ldB, double beta, X_T * X_out, Int ldX, Int nrhs = 1 )
    {
        Check( tb_chol_solve_ex( h_, alpha, B, ldB, detail::dtype_of<B_T>(), beta, X_out, ldX, detail::dtype_of<X_T>(), nrhs ) );
    }
    // X_out = A^{-1} B, Solve.hpp:87-99.
    template<typename B_T, typename X_T>
    void Solve( const B_T * B, X_T * X_out, Int nrhs = 1 )
    {
        Solve( 1.0, B, nrhs, 0.0, X_out, nrhs, nrhs );
    }
    // Same on device buffers of the handle's GPU and stream.
    template<typename B_T, typename X_T>
    void Solve_Device( double alpha, const B_T * d_B, Int ldB, double beta, X_T * d_X, Int ldX, Int nrhs = 1 )
    {
        Check( tb_chol_solve_device_ex( h_, alpha, d_B, ldB, detail::dtype_of<B_T>(), beta, d_X, ldX, detail::dtype_of<X_T>(), nrhs ) );
    }

    // X_out = alpha * P^T U^{-1} P B + beta * X_out (Solve.hpp:182-245).
    void UpperSolve( double alpha, const double * B, Int ldB, double beta, double * X_out, Int ldX, Int nrhs = 1 )
    {
        Check( tb_chol_upper_solve( h_, alpha, B, ldB, beta, X_out, ldX, nrhs ) );
    }
    // X_out = alpha * P^T U^{-T} P B + beta * X_out (Solve.hpp:251-310, documented meaning).
    void LowerSolve( double alpha, const double * B, Int ldB, double beta, double * X_out, Int ldX, Int nrhs = 1 )
    {
        Check( tb_chol_lower_solve( h_, alpha, B, ldB, beta, X_out, ldX, nrhs ) );
    }

    // Conjugate gradients on (A' + reg I) X = B preconditioned by this factor,
    // the reference's ConjugateGradient::operator() (ConjugateGradient.hpp:109)
    // with P = this factor's solve: X_out = alpha x + beta X_out.  A_val: A' in
    // the caller's CSR order (nullptr: the factored values).  Returns whether
    // every column met the relative tolerance; IterationCount() tells the steps.
    bool ConjugateGradient( const double * A_val, double reg, double alpha, const double * B, Int ldB, double beta,
                            double * X_out, Int ldX, Int nrhs, double relative_tolerance, Int max_iter,
                            bool use_initial_guess = false )
    {
        relres_.assign( static_cast<size_t>( nrhs < 1 ? 1 : nrhs ), 0.0 );
        const int st = tb_chol_cg( h_, A_val, reg, alpha, B, ldB, beta, X_out, ldX, nrhs, relative_tolerance, max_iter,
                                   use_initial_guess ? 1 : 0, &cg_iter_, relres_.data() );
        if( st == TB_ERR_NOT_CONVERGED ) { return false; }
        Check( st );
        return true;
    }
    // GMRES on (A' + reg I) X = B preconditioned from the left by this factor,
    // the reference's GMRES::operator() (GMRES.hpp:124-330): max_iter Arnoldi
    // steps per restart, at most max_restarts restarts.  Returns whether every
    // column met |P r| <= relative_tolerance |P b|.
    bool GMRES( const double * A_val, double reg, double alpha, const double * B, Int ldB, double beta,
                double * X_out, Int ldX, Int nrhs, double relative_tolerance, Int max_iter, Int max_restarts,
                bool use_initial_guess = false )
    {
        relres_.assign( static_cast<size_t>( nrhs < 1 ? 1 : nrhs ), 0.0 );
        const int st = tb_chol_gmres( h_, A_val, reg, alpha, B, ldB, beta, X_out, ldX, nrhs, relative_tolerance, max_iter,
                                      max_restarts, use_initial_guess ? 1 : 0, &cg_iter_, &restarts_, relres_.data() );
        if( st == TB_ERR_NOT_CONVERGED ) { return false; }
        Check( st );
        return true;
    }
    Int RestartCount() const { return restarts_; }
    Int IterationCount() const { return cg_iter_; }
    const std::vector<double> & RelativeResiduals() const { return relres_; }

    // Queries, CholeskyDecomposition/InputOutput.hpp:85-367 and Numeric.hpp:183-215.
    Int RowCount() const { Int v = 0; Check( tb_chol_row_count( h_, &v ) ); return v; }
    Int ColCount() const { return RowCount(); }
    LInt NonzeroCount() const { LInt v = 0; Check( tb_chol_nonzero_count( h_, &v ) ); return v; }
    Int SN_Count() const { Int v = 0; Check( tb_chol_sn_count( h_, &v ) ); return v; }

    bool NumericallyFactorizedQ() const { int32_t f = 0, g = 0; Check( tb_chol_factorized( h_, &f, &g ) ); return f != 0; }
    bool NumericallyGoodQ() const { int32_t f = 0, g = 0; Check( tb_chol_factorized( h_, &f, &g ) ); return g != 0; }
    Int FailedSupernode() const { Int v = -1; Check( tb_chol_failed_supernode( h_, &v ) ); return v; }

    LInt RequiredTriangularSize() const { LInt t = 0, r = 0; Check( tb_chol_factor_sizes( h_, &t, &r ) ); return t; }
    LInt RequiredRectangularSize() const { LInt t = 0, r = 0; Check( tb_chol_factor_sizes( h_, &t, &r ) ); return r; }

    std::vector<Int>  SN_RowPointers() const       { return Array<Int>( TB_ARRAY_SN_RP ); }
    std::vector<LInt> SN_Outer() const             { return Array<LInt>( TB_ARRAY_SN_OUTER ); }
    std::vector<Int>  SN_Inner() const             { return Array<Int>( TB_ARRAY_SN_INNER ); }
    std::vector<Int>  RowToSN() const              { return Array<Int>( TB_ARRAY_ROW_TO_SN ); }
    std::vector<LInt> SN_TrianglePointers() const  { return Array<LInt>( TB_ARRAY_SN_TRI_PTR ); }
    std::vector<LInt> SN_RectanglePointers() const { return Array<LInt>( TB_ARRAY_SN_REC_PTR ); }
    std::vector<Int>  Permutation() const          { return Array<Int>( TB_ARRAY_PERM ); }
    std::vector<Int>  InversePermutation() const   { return Array<Int>( TB_ARRAY_PERM_INV ); }
    std::vector<LInt> ValuePermutation() const     { return Array<LInt>( TB_ARRAY_VALUE_PERM ); }

    // GetPermutation / GetValuePermutation (InputOutput.hpp:304-312) under the
    // reference's names: the permutation after postordering as an object with
    // the accessors its callers use, and A's value permutation.
    struct Permutation_T
    {
        std::vector<Int> p, p_inv;
        const std::vector<Int> & GetPermutation() const { return p; }
        const std::vector<Int> & GetInversePermutation() const { return p_inv; }
    };
    Permutation_T GetPermutation() const { return Permutation_T{ Permutation(), InversePermutation() }; }
    std::vector<LInt> GetValuePermutation() const { return ValuePermutation(); }
    std::vector<Int>  AssemblyTreeParents() const  { return Array<Int>( TB_ARRAY_ATREE_PARENTS ); }
    std::vector<Int>  EliminationTreeParents() const { return Array<Int>( TB_ARRAY_ETREE_PARENTS ); }

    // SN_TriangleValues / SN_RectangleValues (InputOutput.hpp:322-352),
    // copied back from the device in the reference's layout.
    std::pair<std::vector<Scal>, std::vector<Scal>> FactorValues() const
    {
        std::vector<double> tri( static_cast<size_t>( RequiredTriangularSize() ) );
        std::vector<double> rec( static_cast<size_t>( RequiredRectangularSize() ) );
        Check( tb_chol_factor_values( h_, tri.data(), rec.data() ) );
        return { std::vector<Scal>( tri.begin(), tri.end() ), std::vector<Scal>( rec.begin(), rec.end() ) };
    }

    // GetU (InputOutput.hpp:116-217): U in the permuted ordering as CSR.
    MatrixCSR GetU() const
    {
        LInt nnz = 0;
        Check( tb_chol_u_nonzero_count( h_, &nnz ) );
        const Int n = RowCount();
        std::vector<LInt> outer( static_cast<size_t>( n ) + 1 );
        std::vector<Int> inner( static_cast<size_t>( nnz ) );
        std::vector<double> values( static_cast<size_t>( nnz ) );
        Check( tb_chol_get_u( h_, outer.data(), inner.data(), values.data() ) );
        return MatrixCSR( outer.data(), inner.data(), values.data(), n, n, 1 );
    }

    // LogDeterminant (InputOutput.hpp:294-297), WriteFactorDiagonal (:238-257).
    Scal LogDeterminant() const { double v = 0; Check( tb_chol_log_det( h_, &v ) ); return static_cast<Scal>( v ); }
    // log det U = half of log det A (InputOutput.hpp:259-292).
    Scal FactorLogDeterminant() const { return static_cast<Scal>( 0.5 ) * LogDeterminant(); }
    void WriteFactorDiagonal( Scal * diag ) const
    {
        std::vector<double> d( static_cast<size_t>( RowCount() ) );
        Check( tb_chol_factor_diagonal( h_, d.data() ) );
        for( size_t i = 0; i < d.size(); ++i ) { diag[i] = static_cast<Scal>( d[i] ); }
    }

    // Stream of the handle (a cudaStream_t).
    void SetStream( void * stream ) { Check( tb_chol_set_stream( h_, stream ) ); }

    tb_chol * Handle() const noexcept { return h_; }

private:
    // Scal = float: FP32 factor storage (the mixed-precision mode)
    void SetScalarPrecision()
    {
        if( std::is_same<Scal, float>::value ) { Check( tb_chol_set_precision( h_, TB_PRECISION_MIXED ) ); }
    }

    template<typename T>
    std::vector<T> Array( int32_t which ) const
    {
        int64_t size = 0;
        Check( tb_chol_array_size( h_, which, &size ) );
        std::vector<int64_t> tmp( static_cast<size_t>( size ) );
        Check( tb_chol_array_copy( h_, which, tmp.data() ) );
        return std::vector<T>( tmp.begin(), tmp.end() );
    }

    tb_chol * h_ = nullptr;
    SupernodeStrategy_T strategy_ = SupernodeStrategy_T::Maximal;     // the reference's defaults
    Int threshold_ = 4;
    FactorizationMethod_T method_ = FactorizationMethod_T::Multifrontal;
    Int threads_ = 1;
    Int cg_iter_ = 0;
    Int restarts_ = 0;
    std::vector<double> relres_;
};

} // namespace Sparse
} // namespace tensors_b200
