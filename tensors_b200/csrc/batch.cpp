// Batched factorization of many independent SPD systems (tb_batch_*).
//
// The systems are placed on the diagonal of one block-diagonal matrix: its
// elimination tree is the forest of the systems' trees, the symbolic
// analysis keeps every system's rows contiguous (the roots are visited in
// ascending order, each subtree is one system's), and the device plan of the
// combined matrix is a merged task list over all systems' supernodes: every
// launch of the level schedule (the default) covers that level and panel step
// of all systems at once, captured in one CUDA graph, so small and large
// systems share the SMs without a launch per system.  The persistent
// task-graph launch over all levels is available through the handle; with
// 400 Delaunay systems it factored in 112 ms against 90 ms for the levels.
#include "tensors_b200.h"
#include "common.hpp"

#include <climits>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

struct tb_batch
{
    tb_chol * h = nullptr;
    std::int32_t count = 0;
    std::vector<std::int64_t> row_off, val_off;     // count + 1 each
    std::vector<double> values;                     // concatenated values for host input
    std::vector<double> rhs, sol;                   // concatenated right-hand sides / solutions
    ~tb_batch() { if( h ) { tb_chol_destroy( h ); } }
};

namespace
{

int bfail( int code, const std::string & msg )
{
    tb::set_last_error( msg );
    return code;
}

} // namespace

extern "C" {

int tb_batch_create( tb_batch ** out, std::int32_t count, const std::int32_t * n, const std::int64_t * const * outer,
                     const std::int32_t * const * inner, const std::int32_t * const * perm, std::int32_t thread_count )
{
    if( out == nullptr || count <= 0 || n == nullptr || outer == nullptr || inner == nullptr )
    {
        return bfail( TB_ERR_INVALID_ARGUMENT, "tb_batch_create: null argument or count <= 0" );
    }
    *out = nullptr;
    tb_batch * b = new tb_batch();
    b->count = count;
    b->row_off.assign( static_cast<size_t>( count ) + 1, 0 );
    b->val_off.assign( static_cast<size_t>( count ) + 1, 0 );
    for( std::int32_t s = 0; s < count; ++s )
    {
        if( n[s] <= 0 || outer[s] == nullptr || inner[s] == nullptr )
        {
            delete b;
            return bfail( TB_ERR_INVALID_ARGUMENT, "tb_batch_create: system " + std::to_string( s ) + " is empty or null" );
        }
        b->row_off[s + 1] = b->row_off[s] + n[s];
        b->val_off[s + 1] = b->val_off[s] + outer[s][n[s]];
    }
    const std::int64_t N = b->row_off[count];
    if( N > INT32_MAX )
    {
        delete b;
        return bfail( TB_ERR_INVALID_ARGUMENT, "tb_batch_create: more than 2^31-1 rows in the batch" );
    }
    std::vector<std::int64_t> outer_c( static_cast<size_t>( N ) + 1 );
    std::vector<std::int32_t> inner_c( static_cast<size_t>( b->val_off[count] ) );
    std::vector<std::int32_t> perm_c( static_cast<size_t>( N ) );
    for( std::int32_t s = 0; s < count; ++s )
    {
        const std::int64_t r0 = b->row_off[s], v0 = b->val_off[s];
        const std::int32_t ns = n[s];
        for( std::int32_t i = 0; i <= ns; ++i ) { outer_c[static_cast<size_t>( r0 + i )] = outer[s][i] + v0; }
        const std::int64_t nnz = outer[s][ns];
        for( std::int64_t e = 0; e < nnz; ++e ) { inner_c[static_cast<size_t>( v0 + e )] = inner[s][e] + static_cast<std::int32_t>( r0 ); }
        for( std::int32_t i = 0; i < ns; ++i )
        {
            const std::int32_t p = (perm && perm[s]) ? perm[s][i] : i;
            perm_c[static_cast<size_t>( r0 + i )] = p + static_cast<std::int32_t>( r0 );
        }
    }
    const int st = tb_chol_create( &b->h, static_cast<std::int32_t>( N ), outer_c.data(), inner_c.data(), perm_c.data(),
                                   thread_count );
    if( st != TB_OK )
    {
        const std::string msg = tb_last_error();
        delete b;
        return bfail( st, "tb_batch_create: " + msg );
    }
    *out = b;
    return TB_OK;
}

int tb_batch_destroy( tb_batch * b )
{
    delete b;
    return TB_OK;
}

int tb_batch_handle( tb_batch * b, tb_chol ** out )
{
    if( b == nullptr || out == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    *out = b->h;
    return TB_OK;
}

int tb_batch_count( tb_batch * b, std::int32_t * out )
{
    if( b == nullptr || out == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    *out = b->count;
    return TB_OK;
}

int tb_batch_offsets( tb_batch * b, std::int64_t * row_offsets, std::int64_t * value_offsets )
{
    if( b == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null batch" ); }
    if( row_offsets ) { std::copy( b->row_off.begin(), b->row_off.end(), row_offsets ); }
    if( value_offsets ) { std::copy( b->val_off.begin(), b->val_off.end(), value_offsets ); }
    return TB_OK;
}

int tb_batch_numeric( tb_batch * b, const double * const * values, double reg )
{
    if( b == nullptr || values == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    b->values.resize( static_cast<size_t>( b->val_off[b->count] ) );
    for( std::int32_t s = 0; s < b->count; ++s )
    {
        if( values[s] == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null values of system " + std::to_string( s ) ); }
        std::memcpy( b->values.data() + b->val_off[s], values[s], sizeof(double) * static_cast<size_t>( b->val_off[s + 1] - b->val_off[s] ) );
    }
    return tb_chol_numeric( b->h, b->values.data(), reg );
}

int tb_batch_numeric_device( tb_batch * b, const double * d_values, double reg )
{
    if( b == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null batch" ); }
    return tb_chol_numeric_device( b->h, d_values, reg );
}

int tb_batch_failed_system( tb_batch * b, std::int32_t * out )
{
    if( b == nullptr || out == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    std::int32_t sn = -1;
    {
        const int st = tb_chol_failed_supernode( b->h, &sn );
        if( st != TB_OK ) { return st; }
    }
    if( sn < 0 ) { *out = -1; return TB_OK; }
    std::int64_t size = 0;
    int st = tb_chol_array_size( b->h, TB_ARRAY_SN_RP, &size );
    if( st != TB_OK ) { return st; }
    std::vector<std::int64_t> rp( static_cast<size_t>( size ) );
    st = tb_chol_array_copy( b->h, TB_ARRAY_SN_RP, rp.data() );
    if( st != TB_OK ) { return st; }
    const std::int64_t row = rp[static_cast<size_t>( sn )];
    *out = static_cast<std::int32_t>( std::upper_bound( b->row_off.begin(), b->row_off.end(), row ) - b->row_off.begin() ) - 1;
    return TB_OK;
}

int tb_batch_solve( tb_batch * b, const double * const * B, double * const * X, std::int32_t nrhs )
{
    if( b == nullptr || B == nullptr || X == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null argument" ); }
    const std::int32_t k = std::max( 1, nrhs );
    const std::int64_t N = b->row_off[b->count];
    b->rhs.resize( static_cast<size_t>( N * k ) );
    b->sol.resize( static_cast<size_t>( N * k ) );
    for( std::int32_t s = 0; s < b->count; ++s )
    {
        if( B[s] == nullptr || X[s] == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null buffer of system " + std::to_string( s ) ); }
        std::memcpy( b->rhs.data() + b->row_off[s] * k, B[s], sizeof(double) * static_cast<size_t>( (b->row_off[s + 1] - b->row_off[s]) * k ) );
    }
    const int st = tb_chol_solve( b->h, 1.0, b->rhs.data(), k, 0.0, b->sol.data(), k, k );
    if( st != TB_OK ) { return st; }
    for( std::int32_t s = 0; s < b->count; ++s )
    {
        std::memcpy( X[s], b->sol.data() + b->row_off[s] * k, sizeof(double) * static_cast<size_t>( (b->row_off[s + 1] - b->row_off[s]) * k ) );
    }
    return TB_OK;
}

int tb_batch_solve_device( tb_batch * b, const double * d_B, double * d_X, std::int32_t nrhs )
{
    if( b == nullptr ) { return bfail( TB_ERR_INVALID_ARGUMENT, "null batch" ); }
    const std::int32_t k = std::max( 1, nrhs );
    return tb_chol_solve_device( b->h, 1.0, d_B, k, 0.0, d_X, k, k );
}

} // extern "C"
