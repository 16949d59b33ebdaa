// MatrixMarket coordinate files <-> CSR on the host.
//
// Reader: MatrixCSR::LoadFromMatrixMarket (src/Sparse/MatrixCSR/MatrixMarket.hpp:3-202)
// followed by the triple assembly it calls, MatrixCSR::FromTriples
// (src/Sparse/MatrixCSR/FromTriples.hpp:4-209) with compression and
// symmetrization on:
//  * banner "%%MatrixMarket matrix coordinate <field> <symmetry>", compared
//    case-insensitively; field real / integer / pattern (pattern entries are
//    1), symmetry general / symmetric; complex, skew-symmetric, hermitian and
//    dense (array) files are rejected, as the reference rejects them;
//  * '%' comment lines, then "rows cols entries", then one 1-based
//    "i j [a]" entry per line;
//  * symmetric files store one triangle: every off-diagonal entry (i, j, a) is
//    also entered as (j, i, a), the diagonal once (FromTriples.hpp:131-145);
//  * the entries of a row keep file order (a mirrored entry follows the entry
//    it mirrors), are sorted by column with a stable sort, and repeated (i, j)
//    pairs are summed in that order (additive assembly, FromTriples.hpp:167-190).
// Unlike the reference (which prints an error and leaves the matrix
// unchanged, or reads past a short file), every failure returns a status:
// TB_ERR_IO for an unreadable file, TB_ERR_FORMAT for a malformed or
// unsupported one (also indices outside the stated size and entry counts
// that differ from the size line).
//
// Writer: MatrixCSR::WriteToMatrixMarket (MatrixMarket.hpp:205-306): a
// "real general" coordinate file, one "%d %d %.17E" line per stored entry in
// CSR order, so a written file reads back bit-exact.

#include "common.hpp"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

int fail( int code, const std::string & msg )
{
    tb::set_last_error( msg );
    return code;
}

int thread_count_or_default( I32 t )
{
    if( t > 0 ) { return t; }
    const unsigned h = std::thread::hardware_concurrency();
    return h == 0 ? 1 : static_cast<int>( std::min( h, 64u ) );
}

template<typename F>
void parallel_for( int threads, F && body )
{
    if( threads <= 1 ) { body( 0 ); return; }
    std::vector<std::thread> pool;
    pool.reserve( static_cast<size_t>( threads ) );
    for( int t = 0; t < threads; ++t ) { pool.emplace_back( [&body, t] { body( t ); } ); }
    for( auto & th : pool ) { th.join(); }
}

bool is_blank( char c ) { return c == ' ' || c == '\t' || c == '\r'; }

const char * skip_blanks( const char * p, const char * end )
{
    while( p < end && is_blank( *p ) ) { ++p; }
    return p;
}

// Text of the file quoted in an error message: printable ASCII only.
std::string quoted( const char * b, const char * e )
{
    std::string s( b, static_cast<size_t>( std::min<std::ptrdiff_t>( e - b, 80 ) ) );
    for( char & c : s ) { if( static_cast<unsigned char>( c ) < 32 || static_cast<unsigned char>( c ) > 126 ) { c = '?'; } }
    return s;
}

std::string lower( std::string s )
{
    for( char & c : s ) { c = static_cast<char>( std::tolower( static_cast<unsigned char>( c ) ) ); }
    return s;
}

template<typename T>
const char * parse_int( const char * p, const char * end, T & out )
{
    p = skip_blanks( p, end );
    if( p < end && *p == '+' ) { ++p; }
    auto r = std::from_chars( p, end, out );
    return r.ec == std::errc() ? r.ptr : nullptr;
}

const char * parse_real( const char * p, const char * end, double & out )
{
    p = skip_blanks( p, end );
    if( p < end && *p == '+' ) { ++p; }
    auto r = std::from_chars( p, end, out, std::chars_format::general );
    return r.ec == std::errc() ? r.ptr : nullptr;
}

struct Chunk
{
    std::vector<I32> i, j;
    std::vector<double> a;
    std::string error;
};

// Parses the entry lines in [begin, end): one entry per line, blank and '%'
// lines skipped.
void parse_entries( const char * begin, const char * end, bool pattern, I32 rows, I32 cols, Chunk & c )
{
    const char * p = begin;
    while( p < end )
    {
        const char * eol = static_cast<const char *>( std::memchr( p, '\n', static_cast<size_t>( end - p ) ) );
        if( eol == nullptr ) { eol = end; }
        const char * q = skip_blanks( p, eol );
        if( q < eol && *q != '%' )
        {
            I64 i = 0, j = 0;
            double a = 1.0;
            q = parse_int( q, eol, i );
            if( q != nullptr ) { q = parse_int( q, eol, j ); }
            if( q != nullptr && !pattern ) { q = parse_real( q, eol, a ); }
            if( q == nullptr )
            {
                c.error = "malformed entry line \"" + quoted( p, eol ) + "\"";
                return;
            }
            if( i < 1 || i > rows || j < 1 || j > cols )
            {
                c.error = "entry (" + std::to_string( i ) + ", " + std::to_string( j ) + ") outside the " + std::to_string( rows )
                          + " x " + std::to_string( cols ) + " matrix";
                return;
            }
            c.i.push_back( static_cast<I32>( i - 1 ) );
            c.j.push_back( static_cast<I32>( j - 1 ) );
            c.a.push_back( a );
        }
        p = eol < end ? eol + 1 : end;
    }
}

bool read_file( const char * path, std::string & text )
{
    std::FILE * f = std::fopen( path, "rb" );
    if( f == nullptr ) { return false; }
    bool ok = std::fseek( f, 0, SEEK_END ) == 0;
    const long size = ok ? std::ftell( f ) : -1;
    ok = ok && size >= 0 && std::fseek( f, 0, SEEK_SET ) == 0;
    if( ok )
    {
        text.resize( static_cast<size_t>( size ) );
        ok = size == 0 || std::fread( &text[0], 1, static_cast<size_t>( size ), f ) == static_cast<size_t>( size );
    }
    std::fclose( f );
    return ok;
}

} // namespace

extern "C" int tb_matrix_market_read( const char * path, int32_t thread_count, int32_t * rows_out, int32_t * cols_out,
                                      int64_t ** outer_out, int32_t ** inner_out, double ** values_out )
{
    if( path == nullptr || rows_out == nullptr || cols_out == nullptr || outer_out == nullptr || inner_out == nullptr
        || values_out == nullptr )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "tb_matrix_market_read: null argument" );
    }
    *outer_out = nullptr; *inner_out = nullptr; *values_out = nullptr;
    std::string text;
    if( !read_file( path, text ) ) { return fail( TB_ERR_IO, std::string( "tb_matrix_market_read: cannot read " ) + path ); }
    const char * p = text.data();
    const char * end = p + text.size();

    // banner
    const char * eol = static_cast<const char *>( std::memchr( p, '\n', text.size() ) );
    if( eol == nullptr ) { eol = end; }
    std::vector<std::string> words;
    for( const char * q = p; q < eol; )
    {
        q = skip_blanks( q, eol );
        const char * w = q;
        while( q < eol && !is_blank( *q ) ) { ++q; }
        if( q > w ) { words.push_back( lower( std::string( w, q ) ) ); }
    }
    if( words.empty() || words[0] != "%%matrixmarket" ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: not a MatrixMarket file" ); }
    if( words.size() < 5 ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: incomplete banner" ); }
    if( words[1] != "matrix" ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: second word of the banner is not \"matrix\"" ); }
    if( words[2] != "coordinate" )
    {
        return fail( TB_ERR_FORMAT, "tb_matrix_market_read: \"" + quoted( words[2].data(), words[2].data() + words[2].size() ) + "\" storage is not supported (coordinate only)" );
    }
    const std::string & field = words[3];
    if( field != "real" && field != "integer" && field != "pattern" && field != "double" )
    {
        return fail( TB_ERR_FORMAT, "tb_matrix_market_read: field \"" + quoted( field.data(), field.data() + field.size() ) + "\" is not supported for real matrices" );
    }
    const bool pattern = field == "pattern";
    const std::string & symmetry = words[4];
    if( symmetry != "general" && symmetry != "symmetric" )
    {
        return fail( TB_ERR_FORMAT, "tb_matrix_market_read: symmetry \"" + quoted( symmetry.data(), symmetry.data() + symmetry.size() ) + "\" is not supported" );
    }
    const bool symmetric = symmetry == "symmetric";

    // comments, then the size line
    p = eol < end ? eol + 1 : end;
    I64 rows = -1, cols = -1, count = -1;
    while( p < end )
    {
        eol = static_cast<const char *>( std::memchr( p, '\n', static_cast<size_t>( end - p ) ) );
        if( eol == nullptr ) { eol = end; }
        const char * q = skip_blanks( p, eol );
        p = eol < end ? eol + 1 : end;
        if( q == eol || *q == '%' ) { continue; }
        q = parse_int( q, eol, rows );
        if( q != nullptr ) { q = parse_int( q, eol, cols ); }
        if( q != nullptr ) { q = parse_int( q, eol, count ); }
        if( q == nullptr ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: malformed size line" ); }
        break;
    }
    if( rows < 0 || cols < 0 || count < 0 ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: missing or negative sizes" ); }
    if( rows > INT32_MAX || cols > INT32_MAX ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: dimensions exceed int32" ); }
    if( symmetric && rows != cols ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: symmetric file with a non-square size" ); }

    // entries: chunks split at line ends, parsed in parallel
    const int threads = std::max( 1, std::min<int>( thread_count_or_default( thread_count ),
                                                    static_cast<int>( (end - p) / (1 << 16) ) + 1 ) );
    std::vector<const char *> cut( static_cast<size_t>( threads ) + 1, end );
    cut[0] = p;
    for( int t = 1; t < threads; ++t )
    {
        const char * c = p + (end - p) * t / threads;
        c = std::max( c, cut[static_cast<size_t>( t ) - 1] );
        const char * nl = static_cast<const char *>( std::memchr( c, '\n', static_cast<size_t>( end - c ) ) );
        cut[static_cast<size_t>( t )] = nl == nullptr ? end : nl + 1;
    }
    std::vector<Chunk> chunk( static_cast<size_t>( threads ) );
    parallel_for( threads, [&]( int t ) {
        parse_entries( cut[static_cast<size_t>( t )], cut[static_cast<size_t>( t ) + 1], pattern, static_cast<I32>( rows ),
                       static_cast<I32>( cols ), chunk[static_cast<size_t>( t )] );
    } );
    I64 found = 0;
    for( const Chunk & c : chunk )
    {
        if( !c.error.empty() ) { return fail( TB_ERR_FORMAT, "tb_matrix_market_read: " + c.error ); }
        found += static_cast<I64>( c.i.size() );
    }
    if( found != count )
    {
        return fail( TB_ERR_FORMAT, "tb_matrix_market_read: the size line declares " + std::to_string( count ) + " entries, the file holds "
                                    + std::to_string( found ) );
    }

    // rows: entries in file order, mirrored entries right after their originals
    const I32 m = static_cast<I32>( rows );
    std::vector<I64> ptr( static_cast<size_t>( m ) + 1, 0 );
    for( const Chunk & c : chunk )
    {
        for( size_t k = 0; k < c.i.size(); ++k )
        {
            ++ptr[static_cast<size_t>( c.i[k] ) + 1];
            if( symmetric && c.i[k] != c.j[k] ) { ++ptr[static_cast<size_t>( c.j[k] ) + 1]; }
        }
    }
    std::partial_sum( ptr.begin(), ptr.end(), ptr.begin() );
    const I64 total = ptr[static_cast<size_t>( m )];
    std::vector<I32> col( static_cast<size_t>( total ) );
    std::vector<double> val( static_cast<size_t>( total ) );
    {
        std::vector<I64> pos( ptr.begin(), ptr.end() - 1 );
        for( const Chunk & c : chunk )
        {
            for( size_t k = 0; k < c.i.size(); ++k )
            {
                I64 & q = pos[static_cast<size_t>( c.i[k] )];
                col[static_cast<size_t>( q )] = c.j[k]; val[static_cast<size_t>( q )] = c.a[k]; ++q;
                if( symmetric && c.i[k] != c.j[k] )
                {
                    I64 & r = pos[static_cast<size_t>( c.j[k] )];
                    col[static_cast<size_t>( r )] = c.i[k]; val[static_cast<size_t>( r )] = c.a[k]; ++r;
                }
            }
        }
    }
    chunk.clear();

    // per row: stable sort by column, sum repeated columns in order
    const int row_threads = std::max( 1, std::min<int>( thread_count_or_default( thread_count ), static_cast<int>( total / (1 << 16) ) + 1 ) );
    std::vector<I64> kept( static_cast<size_t>( m ), 0 );
    parallel_for( row_threads, [&]( int t ) {
        const I32 r0 = static_cast<I32>( static_cast<I64>( m ) * t / row_threads );
        const I32 r1 = static_cast<I32>( static_cast<I64>( m ) * (t + 1) / row_threads );
        std::vector<I64> order;
        std::vector<I32> c2;
        std::vector<double> v2;
        for( I32 r = r0; r < r1; ++r )
        {
            const I64 b = ptr[static_cast<size_t>( r )], e = ptr[static_cast<size_t>( r ) + 1];
            if( e == b ) { continue; }
            order.resize( static_cast<size_t>( e - b ) );
            std::iota( order.begin(), order.end(), b );
            std::stable_sort( order.begin(), order.end(), [&]( I64 x, I64 y ) { return col[static_cast<size_t>( x )] < col[static_cast<size_t>( y )]; } );
            c2.clear(); v2.clear();
            for( I64 k : order )
            {
                if( !c2.empty() && c2.back() == col[static_cast<size_t>( k )] ) { v2.back() += val[static_cast<size_t>( k )]; }
                else { c2.push_back( col[static_cast<size_t>( k )] ); v2.push_back( val[static_cast<size_t>( k )] ); }
            }
            std::copy( c2.begin(), c2.end(), col.begin() + b );
            std::copy( v2.begin(), v2.end(), val.begin() + b );
            kept[static_cast<size_t>( r )] = static_cast<I64>( c2.size() );
        }
    } );
    I64 nnz = 0;
    for( I32 r = 0; r < m; ++r ) { nnz += kept[static_cast<size_t>( r )]; }

    int64_t * outer = static_cast<int64_t *>( std::malloc( sizeof( int64_t ) * (static_cast<size_t>( m ) + 1) ) );
    int32_t * inner = static_cast<int32_t *>( std::malloc( sizeof( int32_t ) * std::max<size_t>( 1, static_cast<size_t>( nnz ) ) ) );
    double * values = static_cast<double *>( std::malloc( sizeof( double ) * std::max<size_t>( 1, static_cast<size_t>( nnz ) ) ) );
    if( outer == nullptr || inner == nullptr || values == nullptr )
    {
        std::free( outer ); std::free( inner ); std::free( values );
        return fail( TB_ERR_OUT_OF_MEMORY, "tb_matrix_market_read: out of host memory" );
    }
    outer[0] = 0;
    for( I32 r = 0; r < m; ++r ) { outer[r + 1] = outer[r] + kept[static_cast<size_t>( r )]; }
    parallel_for( row_threads, [&]( int t ) {
        const I32 r0 = static_cast<I32>( static_cast<I64>( m ) * t / row_threads );
        const I32 r1 = static_cast<I32>( static_cast<I64>( m ) * (t + 1) / row_threads );
        for( I32 r = r0; r < r1; ++r )
        {
            const I64 b = ptr[static_cast<size_t>( r )], k = kept[static_cast<size_t>( r )];
            std::copy( col.begin() + b, col.begin() + b + k, inner + outer[r] );
            std::copy( val.begin() + b, val.begin() + b + k, values + outer[r] );
        }
    } );
    *rows_out = m;
    *cols_out = static_cast<I32>( cols );
    *outer_out = outer; *inner_out = inner; *values_out = values;
    return TB_OK;
}

extern "C" int tb_matrix_market_free( void * p )
{
    std::free( p );
    return TB_OK;
}

extern "C" int tb_matrix_market_write( const char * path, int32_t rows, int32_t cols, const int64_t * outer,
                                       const int32_t * inner, const double * values )
{
    if( path == nullptr || rows < 0 || cols < 0 || outer == nullptr ) { return fail( TB_ERR_INVALID_ARGUMENT, "tb_matrix_market_write: bad argument" ); }
    const I64 nnz = outer[rows];
    if( outer[0] != 0 || nnz < 0 || (nnz > 0 && (inner == nullptr || values == nullptr)) )
    {
        return fail( TB_ERR_INVALID_ARGUMENT, "tb_matrix_market_write: malformed CSR" );
    }
    for( I32 r = 0; r < rows; ++r )
    {
        if( outer[r + 1] < outer[r] ) { return fail( TB_ERR_INVALID_ARGUMENT, "tb_matrix_market_write: row pointers decrease" ); }
    }
    for( I64 k = 0; k < nnz; ++k )
    {
        if( inner[k] < 0 || inner[k] >= cols ) { return fail( TB_ERR_INVALID_ARGUMENT, "tb_matrix_market_write: column index out of range" ); }
    }
    // rows formatted in parallel slices, written in order
    const int threads = std::max( 1, std::min<int>( thread_count_or_default( 0 ), static_cast<int>( nnz / (1 << 15) ) + 1 ) );
    std::vector<std::string> part( static_cast<size_t>( threads ) );
    parallel_for( threads, [&]( int t ) {
        const I32 r0 = static_cast<I32>( static_cast<I64>( rows ) * t / threads );
        const I32 r1 = static_cast<I32>( static_cast<I64>( rows ) * (t + 1) / threads );
        std::string & s = part[static_cast<size_t>( t )];
        char line[96];
        for( I32 r = r0; r < r1; ++r )
        {
            for( I64 k = outer[r]; k < outer[r + 1]; ++k )
            {
                const int len = std::snprintf( line, sizeof( line ), "%d %d %.17E\n", r + 1, inner[k] + 1, values[k] );
                s.append( line, static_cast<size_t>( len ) );
            }
        }
    } );
    std::FILE * f = std::fopen( path, "wb" );
    if( f == nullptr ) { return fail( TB_ERR_IO, std::string( "tb_matrix_market_write: cannot open " ) + path ); }
    const std::string head = "%%MatrixMarket matrix coordinate real general\n" + std::to_string( rows ) + " " + std::to_string( cols ) + " "
                             + std::to_string( nnz ) + "\n";
    bool ok = std::fwrite( head.data(), 1, head.size(), f ) == head.size();
    for( const std::string & s : part ) { ok = ok && std::fwrite( s.data(), 1, s.size(), f ) == s.size(); }
    ok = (std::fclose( f ) == 0) && ok;
    return ok ? TB_OK : fail( TB_ERR_IO, std::string( "tb_matrix_market_write: write failed for " ) + path );
}
