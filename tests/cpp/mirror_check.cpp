// Exercises the C++ mirror class (include/tensors_b200/CholeskyDecomposition.hpp)
// the way a user of the reference's Sparse::CholeskyDecomposition would:
// 2D 5-point Laplacian on a g x g grid (+ shift), reversed ordering as the
// fill-reducing permutation, symbolic phase, and with "numeric" as second
// argument a factorization and a 3-RHS solve whose relative residual is
// printed.  Output: "sn_count <S>" [ "status <0|1>" "relres <r>" ].
// "mm <in> <out>": MatrixCSR::LoadFromMatrixMarket of <in>, a Cholesky
// symbolic phase on its pattern, WriteToMatrixMarket to <out>; prints
// "rows <m> nnz <k> sn_count <S>".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tensors_b200/CholeskyDecomposition.hpp"
#include "tensors_b200/MatrixCSR.hpp"

// the reference driver's instantiation (Example_SparseCholesky/main.cpp:31-32)
using CholeskyDecomposition = tensors_b200::Sparse::CholeskyDecomposition<double, int32_t, int64_t>;
using CholeskyDecompositionF = tensors_b200::Sparse::CholeskyDecomposition<float, int32_t, int64_t>;
using tensors_b200::Sparse::MatrixCSR;

int main( int argc, char ** argv )
{
    if( argc > 3 && std::string( argv[1] ) == "mm" )
    {
        MatrixCSR A;
        A.LoadFromMatrixMarket( argv[2], 4 );
        CholeskyDecomposition S( A.Outer().data(), A.Inner().data(), A.RowCount(), 1 );
        S.SymbolicFactorization();
        A.WriteToMatrixMarket( argv[3] );
        std::printf( "rows %d nnz %lld sn_count %d\n", A.RowCount(), static_cast<long long>( A.NonzeroCount() ), S.SN_Count() );
        return 0;
    }
    const int g = argc > 1 ? std::atoi( argv[1] ) : 20;
    const bool numeric = argc > 2 && std::string( argv[2] ) == "numeric";
    const int n = g * g;
    std::vector<int64_t> outer( 1, 0 );
    std::vector<int32_t> inner;
    std::vector<double> val;
    for( int i = 0; i < g; ++i )
    {
        for( int j = 0; j < g; ++j )
        {
            const int r = i * g + j;
            auto add = [&]( int c, double v ) { inner.push_back( c ); val.push_back( v ); };
            if( i > 0 )     { add( r - g, -1.0 ); }
            if( j > 0 )     { add( r - 1, -1.0 ); }
            add( r, 4.0 + 1e-2 );
            if( j + 1 < g ) { add( r + 1, -1.0 ); }
            if( i + 1 < g ) { add( r + g, -1.0 ); }
            outer.push_back( static_cast<int64_t>( inner.size() ) );
        }
    }
    std::vector<int32_t> p( n );
    for( int i = 0; i < n; ++i ) { p[i] = n - 1 - i; }

    CholeskyDecomposition S( outer.data(), inner.data(), p.data(), n, 1 );
    S.SymbolicFactorization();
    std::printf( "sn_count %d\n", S.SN_Count() );
    // the reference's accessor shapes: S.GetPermutation().GetPermutation() and its inverse
    const auto P = S.GetPermutation();
    for( int i = 0; i < n; ++i ) { if( P.GetInversePermutation()[P.GetPermutation()[i]] != i ) { return 2; } }
    if( static_cast<int64_t>( S.GetValuePermutation().size() ) != S.NonzeroCount() ) { return 3; }
    // settings read back with the reference's getters, and across a move
    S.SetAmalgamationThreshold( 4 );
    CholeskyDecomposition T( std::move( S ) );
    if( T.AmalgamationThreshold() != 4 || T.ThreadCount() != 1
        || T.GetSupernodeStrategy() != tensors_b200::Sparse::SupernodeStrategy_T::Maximal
        || T.GetFactorizationMethod() != tensors_b200::Sparse::FactorizationMethod_T::Multifrontal ) { return 4; }
    S = std::move( T );
    if( !numeric ) { return 0; }

    const int status = S.NumericFactorization( val.data(), 0.0 );
    std::printf( "status %d\n", status );
    const int nrhs = 3;
    std::vector<double> B( static_cast<size_t>( n ) * nrhs ), X( B.size() );
    for( size_t k = 0; k < B.size(); ++k ) { B[k] = std::sin( 0.37 * static_cast<double>( k ) ); }
    S.Solve( B.data(), X.data(), nrhs );
    double rn = 0.0, bn = 0.0;
    for( int r = 0; r < n; ++r )
    {
        for( int k = 0; k < nrhs; ++k )
        {
            double ax = 0.0;
            for( int64_t l = outer[r]; l < outer[r + 1]; ++l ) { ax += val[l] * X[inner[l] * nrhs + k]; }
            const double d = B[r * nrhs + k] - ax;
            rn += d * d;
            bn += B[r * nrhs + k] * B[r * nrhs + k];
        }
    }
    std::printf( "relres %.3e\n", std::sqrt( rn / bn ) );
    // conjugate gradients on the unshifted matrix, preconditioned by the shifted factor
    std::vector<double> val2( val );
    for( int r = 0; r < n; ++r )
    {
        for( int64_t l = outer[r]; l < outer[r + 1]; ++l ) { if( inner[l] == r ) { val2[l] -= 5e-3; } }
    }
    const bool ok = S.ConjugateGradient( val2.data(), 0.0, 1.0, B.data(), nrhs, 0.0, X.data(), nrhs, nrhs, 1e-12, 200 );
    std::printf( "cg_ok %d\ncg_iter %d\n", ok ? 1 : 0, S.IterationCount() );
    const bool gok = S.GMRES( val2.data(), 0.0, 1.0, B.data(), nrhs, 0.0, X.data(), nrhs, nrhs, 1e-12, 30, 10 );
    std::printf( "gmres_ok %d\ngmres_iter %d\n", gok ? 1 : 0, S.IterationCount() );

    // relative residual of Y for the matrix with values vv
    auto relres_of = [&]( const std::vector<double> & vv, const std::vector<double> & Y ) {
        double r2 = 0.0, b2 = 0.0;
        for( int r = 0; r < n; ++r )
        {
            for( int k = 0; k < nrhs; ++k )
            {
                double ax = 0.0;
                for( int64_t l = outer[r]; l < outer[r + 1]; ++l ) { ax += vv[l] * Y[inner[l] * nrhs + k]; }
                const double d = B[r * nrhs + k] - ax;
                r2 += d * d;
                b2 += B[r * nrhs + k] * B[r * nrhs + k];
            }
        }
        return std::sqrt( r2 / b2 );
    };
    // float right-hand sides, double solution (cast on copy, Solve.hpp:20-27)
    std::vector<float> Bf( B.begin(), B.end() );
    std::vector<double> Xd( B.size() );
    S.Solve( Bf.data(), Xd.data(), nrhs );
    double rn2 = 0.0, bn2 = 0.0;
    for( int r = 0; r < n; ++r )
    {
        for( int k = 0; k < nrhs; ++k )
        {
            double ax = 0.0;
            for( int64_t l = outer[r]; l < outer[r + 1]; ++l ) { ax += val[l] * Xd[inner[l] * nrhs + k]; }
            const double d = static_cast<double>( Bf[r * nrhs + k] ) - ax;
            rn2 += d * d;
            bn2 += static_cast<double>( Bf[r * nrhs + k] ) * Bf[r * nrhs + k];
        }
    }
    std::printf( "relres_f32_in %.3e\n", std::sqrt( rn2 / bn2 ) );

    // Scal = float: FP32 factor of float values, solves refined against those values (as FP64)
    CholeskyDecompositionF F( outer.data(), inner.data(), p.data(), n, 1 );
    std::vector<float> valf( val.begin(), val.end() );
    std::printf( "status_f32 %d\n", F.NumericFactorization( valf.data(), 0.0f ) );
    std::vector<double> Xf( B.size() );
    F.Solve( B.data(), Xf.data(), nrhs );
    std::printf( "relres_f32_factor %.3e\n", relres_of( std::vector<double>( valf.begin(), valf.end() ), Xf ) );

    // SwapNumericalFactorization: S's factor moves to a second decomposition of the same pattern
    CholeskyDecomposition S2( outer.data(), inner.data(), p.data(), n, 1 );
    CholeskyDecomposition::NumericalFactorization_T cont;
    S.SwapNumericalFactorization( cont );
    const bool moved = cont.NumericallyFactorizedQ() && cont.NumericallyGoodQ() && !S.NumericallyFactorizedQ();
    S2.SwapNumericalFactorization( cont );
    std::vector<double> X2( B.size() );
    S2.Solve( B.data(), X2.data(), nrhs );
    std::printf( "swap_moved %d\nrelres_swapped %.3e\n", moved ? 1 : 0, relres_of( val, X2 ) );
    return 0;
}
