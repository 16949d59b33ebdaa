// tensors_b200::Sparse::MatrixCSR -- the file input and output of
// Tensors::Sparse::MatrixCSR<double,int32_t,int64_t> (src/Sparse/MatrixCSR.hpp)
// over the C-ABI of tensors_b200.h: LoadFromMatrixMarket and
// WriteToMatrixMarket (src/Sparse/MatrixCSR/MatrixMarket.hpp:3, :205) with the
// CSR accessors the Cholesky constructor takes its pattern from.
//
// Differences: errors throw tensors_b200::Sparse::Error (the reference prints
// and leaves the matrix unchanged); repeated entries are summed in file order
// (the reference's order is that of an unstable sort); the writer emits every
// row (the reference's merges two of its four slices, MatrixMarket.hpp:296-305).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <vector>

#include "../tensors_b200.h"
#include "Error.hpp"

namespace tensors_b200 {
namespace Sparse {

class MatrixCSR
{
public:
    using Scal = double;
    using Int  = int32_t;
    using LInt = int64_t;

    MatrixCSR() : outer_( 1, 0 ) {}

    MatrixCSR( const LInt * outer, const Int * inner, const Scal * values, Int m, Int n, Int thread_count = 1 )
    :   m_( m ), n_( n ), threads_( thread_count ),
        outer_( outer, outer + m + 1 ), inner_( inner, inner + outer[m] ), values_( values, values + outer[m] )
    {}

    void LoadFromMatrixMarket( const std::filesystem::path & file, Int thread_count )
    {
        Int m = 0, n = 0;
        LInt * o = nullptr; Int * i = nullptr; Scal * v = nullptr;
        Check( tb_matrix_market_read( file.string().c_str(), thread_count, &m, &n, &o, &i, &v ) );
        const LInt nnz = o[m];
        outer_.assign( o, o + m + 1 );
        inner_.assign( i, i + nnz );
        values_.assign( v, v + nnz );
        tb_matrix_market_free( o ); tb_matrix_market_free( i ); tb_matrix_market_free( v );
        m_ = m; n_ = n; threads_ = thread_count;
    }

    void WriteToMatrixMarket( const std::filesystem::path & file ) const
    {
        Check( tb_matrix_market_write( file.string().c_str(), m_, n_, outer_.data(), inner_.data(), values_.data() ) );
    }

    Int  RowCount()     const { return m_; }
    Int  ColCount()     const { return n_; }
    LInt NonzeroCount() const { return outer_.back(); }
    Int  ThreadCount()  const { return threads_; }
    const std::vector<LInt> & Outer()  const { return outer_; }
    const std::vector<Int>  & Inner()  const { return inner_; }
    const std::vector<Scal> & Values() const { return values_; }

private:
    Int m_ = 0, n_ = 0, threads_ = 1;
    std::vector<LInt> outer_;
    std::vector<Int>  inner_;
    std::vector<Scal> values_;
};

} // namespace Sparse
} // namespace tensors_b200
