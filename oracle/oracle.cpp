// CPU restatement of the reference's supernodal Cholesky path.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py as the checker.  The product never uses it.
//
// Every function below restates one piece of HenrikSchumacher/Tensors'
// Sparse::CholeskyDecomposition<double,int32,int64> in plain sequential C++
// and cites the reference lines it follows.  Dense kernels (potrf, trsm, syrk)
// are textbook loops in the same row-major-U layout the reference stores.

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace
{
using I32 = std::int32_t;
using I64 = std::int64_t;

struct Oracle
{
    I32 n = 0;
    std::vector<I32> p, pinv;                 // row/column permutation
    std::vector<I64> outer;                   // permuted pattern
    std::vector<I32> inner;
    std::vector<I64> vperm;                   // nonzero-value permutation
    std::vector<I64> diag;                    // first entry >= row index

    std::vector<I32> eparent;                 // elimination tree, root = n
    std::vector<I32> echild_ptr, echild_idx;
    std::vector<I32> edesc;                   // descendant counts (n+1)

    I32 sn_count = 0;
    std::vector<I32> sn_rp;
    std::vector<I64> sn_outer;
    std::vector<I32> sn_inner;
    std::vector<I32> row_to_sn;
    std::vector<I64> tri_ptr, rec_ptr;
    I32 max_n0 = 0, max_n1 = 0;

    std::vector<I32> aparent, achild_ptr, achild_idx;

    std::vector<double> aval, tri, rec;
    bool good = false;
};

// Permutation.hpp:828-930 (permutePatternCSR with sorting): row i of the
// result is row p[i] of the input, column j becomes pinv[j], rows are sorted
// and the returned array maps each new nonzero to its old position.
std::vector<I64> permute_pattern( std::vector<I64> & outer, std::vector<I32> & inner,
                                  const std::vector<I32> & p, const std::vector<I32> & pinv )
{
    const I32 m = static_cast<I32>(p.size());
    const I64 nnz = static_cast<I64>(inner.size());
    std::vector<I64> new_outer( static_cast<size_t>(m) + 1, 0 );
    std::vector<I32> new_inner( static_cast<size_t>(nnz) );
    std::vector<I64> perm( static_cast<size_t>(nnz) );
    for( I32 i = 0; i < m; ++i ) { new_outer[i+1] = outer[p[i]+1] - outer[p[i]]; }
    for( I32 i = 0; i < m; ++i ) { new_outer[i+1] += new_outer[i]; }
    std::vector<std::pair<I32,I64>> row;
    for( I32 i = 0; i < m; ++i )
    {
        const I64 begin = outer[p[i]];
        const I64 len   = new_outer[i+1] - new_outer[i];
        row.resize( static_cast<size_t>(len) );
        for( I64 k = 0; k < len; ++k ) { row[k] = { pinv[inner[begin+k]], begin + k }; }
        std::sort( row.begin(), row.end() );
        for( I64 k = 0; k < len; ++k )
        {
            new_inner[new_outer[i]+k] = row[k].first;
            perm     [new_outer[i]+k] = row[k].second;
        }
    }
    outer.swap( new_outer );
    inner.swap( new_inner );
    return perm;
}

// PatternCSR.hpp:408-445 (RequireDiag): first entry of each row whose column
// is >= the row index.
void require_diag( Oracle & o )
{
    o.diag.assign( static_cast<size_t>(o.n), 0 );
    for( I32 i = 0; i < o.n; ++i )
    {
        I64 k = o.outer[i];
        while( k < o.outer[i+1] && o.inner[k] < i ) { ++k; }
        o.diag[i] = k;
    }
}

// EliminationTreeParents.hpp:8-63: elimination tree by path compression
// (Scott & Tuma, Alg. 4.2); roots get parent n.
void elimination_tree( Oracle & o )
{
    const I32 n = o.n;
    o.eparent.assign( static_cast<size_t>(n), n );
    std::vector<I32> a( static_cast<size_t>(n), n );
    for( I32 k = 1; k < n; ++k )
    {
        for( I64 l = o.outer[k]; l < o.outer[k+1]; ++l )
        {
            I32 i = o.inner[l];
            while( (i != n) && (i < k) )
            {
                const I32 j = a[i];
                a[i] = k;
                if( j == n ) { o.eparent[i] = k; }
                i = j;
            }
        }
    }
}

// Tree.hpp:66-91 + Tree/Init.hpp:5-167: a rooted forest over vertices
// [0,count) plus the virtual root `count`, children sorted ascending (the
// adjacency matrix is assembled from (parent, child) pairs and row-sorted,
// PatternCSR/FromPairs.hpp).  Postorder by the iterative DFS of
// Tree/Traverse_PostOrdered_Sequential.hpp:4-71 (children pushed in reverse,
// :40-44); the virtual root is left out of the ordering (Init.hpp:92-97).
void build_tree( const std::vector<I32> & parent, std::vector<I32> & child_ptr,
                 std::vector<I32> & child_idx, std::vector<I32> * post, std::vector<I32> * desc )
{
    const I32 count = static_cast<I32>(parent.size());
    const I32 nv = count + 1;
    child_ptr.assign( static_cast<size_t>(nv) + 1, 0 );
    for( I32 i = 0; i < count; ++i ) { ++child_ptr[parent[i]+1]; }
    for( I32 v = 0; v < nv; ++v ) { child_ptr[v+1] += child_ptr[v]; }
    child_idx.assign( static_cast<size_t>(count), 0 );
    std::vector<I32> fill( child_ptr.begin(), child_ptr.end() - 1 );
    for( I32 i = 0; i < count; ++i ) { child_idx[fill[parent[i]]++] = i; }   // ascending by construction

    if( post == nullptr && desc == nullptr ) { return; }

    std::vector<I32> stack( static_cast<size_t>(nv) ), seen( static_cast<size_t>(nv), 0 );
    std::vector<I32> d( static_cast<size_t>(nv), 0 );
    std::vector<I32> order;
    order.reserve( static_cast<size_t>(count) );
    I32 top = 0;
    stack[0] = count;
    while( top >= 0 )
    {
        const I32 node = stack[top];
        const I32 kb = child_ptr[node], ke = child_ptr[node+1];
        if( !seen[top] && kb < ke )
        {
            seen[top] = 1;
            for( I32 k = ke; k-- > kb; ) { stack[++top] = child_idx[k]; seen[top] = 0; }
        }
        else
        {
            seen[top--] = 0;
            if( node != count ) { order.push_back( node ); }
            I32 sum = 0;
            for( I32 k = kb; k < ke; ++k ) { sum += d[child_idx[k]] + 1; }
            d[node] = sum;
        }
    }
    if( post ) { *post = order; }
    if( desc ) { *desc = d; }
}

// Tree.hpp:264-286 (PostOrderedQ).
bool post_ordered( const std::vector<I32> & parent, const std::vector<I32> & desc )
{
    const I32 count = static_cast<I32>(parent.size());
    for( I32 i = 0; i < count; ++i )
    {
        const I32 pi = parent[i];
        if( !( (i < pi) && (static_cast<I64>(i) + desc[pi] >= static_cast<I64>(pi) + desc[i]) ) ) { return false; }
    }
    return true;
}

void etree_and_children( Oracle & o, std::vector<I32> * post )
{
    elimination_tree( o );
    build_tree( o.eparent, o.echild_ptr, o.echild_idx, post, &o.edesc );
}

// CholeskyDecomposition.hpp:427-472 (PostOrdering): if the elimination tree
// is not postordered, compose the permutation with its postorder
// (Permutation.hpp:294-375, Compose::Post: p[i] <- p[post[i]]), permute the
// pattern again and compose the value permutation (:447-451).
void post_ordering( Oracle & o )
{
    std::vector<I32> post;
    etree_and_children( o, &post );
    if( post_ordered( o.eparent, o.edesc ) ) { return; }

    std::vector<I32> post_inv( post.size() );
    for( I32 i = 0; i < o.n; ++i ) { post_inv[post[i]] = i; }

    std::vector<I32> np( o.p.size() ), npinv( o.p.size() );
    for( I32 i = 0; i < o.n; ++i ) { np[i] = o.p[post[i]]; }
    for( I32 i = 0; i < o.n; ++i ) { npinv[np[i]] = i; }
    o.p.swap( np );
    o.pinv.swap( npinv );

    std::vector<I64> q = permute_pattern( o.outer, o.inner, post, post_inv );
    for( size_t i = 0; i < q.size(); ++i ) { q[i] = o.vperm[q[i]]; }
    o.vperm.swap( q );
    require_diag( o );
    etree_and_children( o, nullptr );
}

// UniteSortedBuffers.hpp:6-163: sorted union without duplicates.
std::vector<I32> unite( const std::vector<I32> & u, const I32 * v, I64 nv )
{
    std::vector<I32> w;
    w.reserve( u.size() + static_cast<size_t>(nv) );
    size_t i = 0; I64 j = 0;
    auto push = [&w]( I32 x ) { if( w.empty() || w.back() != x ) { w.push_back( x ); } };
    while( i < u.size() && j < nv ) { if( u[i] <= v[j] ) { push( u[i++] ); } else { push( v[j++] ); } }
    while( i < u.size() ) { push( u[i++] ); }
    while( j < nv ) { push( v[j++] ); }
    return w;
}

// Symbolic.hpp:590-622 (FundamentalQ, Liu-Ng-Peyton Thm 2.3 / Cor 3.2 as
// the reference implements it: a row with more than one child returns early,
// without recording its columns in prev_col_nz).
bool fundamental( Oracle & o, I32 i, std::vector<I32> & prev_col_nz )
{
    bool is_fund = (i == o.n);
    is_fund = is_fund || ( (o.echild_ptr[i+1] - o.echild_ptr[i]) > 1 );
    if( !is_fund )
    {
        const I32 threshold = i - o.edesc[i] + 1;
        for( I64 k = o.diag[i] + 1; k < o.outer[i+1]; ++k )
        {
            const I32 j = o.inner[k];
            const I32 l = prev_col_nz[j];
            prev_col_nz[j] = i;
            is_fund = is_fund || (l < threshold);
        }
    }
    return is_fund;
}

// Symbolic.hpp:71-256 (Amalgamated), :258-445 (Maximal), :447-588
// (Fundamental): one pass over the rows; a fundamental row closes the
// current supernode, whose column set is the upper pattern of its first row
// beyond the supernode merged with its elimination-tree children's sets.
// Maximal merges a closed supernode into its predecessor when their trailing
// column sets agree; Amalgamated merges while the joint row count stays
// within the threshold.
void find_supernodes( Oracle & o, int strategy, I32 threshold )
{
    const I32 n = o.n;
    std::vector<I32> prev_col_nz( static_cast<size_t>(n), -1 );
    o.row_to_sn.assign( static_cast<size_t>(n), 0 );
    o.sn_rp.assign( static_cast<size_t>(n) + 2, 0 );
    o.sn_outer.assign( static_cast<size_t>(n) + 2, 0 );
    std::vector<I32> agg;   // SN_inner under construction (Aggregator)

    I32 sn = 0, curr_n0 = 0, curr_i0 = 0, prev_n0 = 0, prev_n1 = 0;
    std::vector<I32> curr;

    for( I32 i = 1; i < n + 1; ++i )
    {
        if( fundamental( o, i, prev_col_nz ) )
        {
            curr_n0 = i - curr_i0;
            {
                I64 k = o.diag[curr_i0] + 1;
                const I64 k_end = o.outer[curr_i0+1];
                while( k < k_end && o.inner[k] < i ) { ++k; }
                curr.assign( o.inner.begin() + k, o.inner.begin() + k_end );
            }
            for( I32 l = o.echild_ptr[curr_i0]; l < o.echild_ptr[curr_i0+1]; ++l )
            {
                const I32 j = o.echild_idx[l];
                const I32 k = o.row_to_sn[j];
                if( k == sn ) { continue; }
                I64 a = o.sn_outer[k];
                const I64 b = o.sn_outer[k+1];
                while( a < b && agg[a] < i ) { ++a; }
                if( a < b ) { curr = unite( curr, &agg[a], b - a ); }
            }

            bool merge = false;
            if( strategy == TB_ORACLE_MAXIMAL && sn > 0 )
            {
                I64 a = o.sn_outer[sn-1];
                const I64 b = o.sn_outer[sn];
                while( a < b && agg[a] < i ) { ++a; }
                const I32 c_n1 = static_cast<I32>(curr.size());
                if( c_n1 > 0 && b - a == static_cast<I64>(c_n1) )
                {
                    merge = std::equal( curr.begin(), curr.end(), agg.begin() + a );
                }
            }
            else if( strategy == TB_ORACLE_AMALGAMATED && sn > 0 && curr_n0 + prev_n0 <= threshold )
            {
                I64 a = o.sn_outer[sn-1];
                const I64 b = o.sn_outer[sn];
                while( a < b && agg[a] < i ) { ++a; }
                if( a < b ) { curr = unite( curr, &agg[a], b - a ); }
                merge = true;
            }
            if( merge )
            {
                --sn;
                agg.resize( agg.size() - static_cast<size_t>(prev_n1) );
                for( I32 k = i - curr_n0; k < i; ++k ) { o.row_to_sn[k] = sn; }
                curr_n0 += prev_n0;
            }

            agg.insert( agg.end(), curr.begin(), curr.end() );
            ++sn;
            o.sn_outer[sn] = static_cast<I64>(agg.size());
            o.sn_rp[sn] = curr_i0 = i;
            prev_n0 = curr_n0;
            prev_n1 = static_cast<I32>(curr.size());
        }
        if( i < n ) { o.row_to_sn[i] = sn; }
    }
    o.sn_count = sn;
    o.sn_rp.resize( static_cast<size_t>(sn) + 1 );
    o.sn_outer.resize( static_cast<size_t>(sn) + 1 );
    o.sn_inner = agg;
}

// Symbolic.hpp:36-60 (pointer prefix sums over full n0 x n0 squares and
// n0 x n1 rectangles) and AssemblyTree.hpp:12-61 (supernode parents).
void finish_symbolic( Oracle & o )
{
    const I32 S = o.sn_count;
    o.tri_ptr.assign( static_cast<size_t>(S) + 1, 0 );
    o.rec_ptr.assign( static_cast<size_t>(S) + 1, 0 );
    o.max_n0 = o.max_n1 = 0;
    for( I32 k = 0; k < S; ++k )
    {
        const I32 n0 = o.sn_rp[k+1] - o.sn_rp[k];
        const I32 n1 = static_cast<I32>( o.sn_outer[k+1] - o.sn_outer[k] );
        o.max_n0 = std::max( o.max_n0, n0 );
        o.max_n1 = std::max( o.max_n1, n1 );
        o.tri_ptr[k+1] = o.tri_ptr[k] + static_cast<I64>(n0) * n0;
        o.rec_ptr[k+1] = o.rec_ptr[k] + static_cast<I64>(n0) * n1;
    }
    o.aparent.assign( static_cast<size_t>(S), S );
    for( I32 k = 0; k + 1 < S; ++k )
    {
        const I32 lp = o.eparent[ o.sn_rp[k+1] - 1 ];
        o.aparent[k] = (lp < o.n) ? o.row_to_sn[lp] : S;
    }
    build_tree( o.aparent, o.achild_ptr, o.achild_idx, nullptr, nullptr );
}

// potrf<RowMajor,Upper> (LAPACK/potrf.hpp:7-93): U^T U = A on the upper
// triangle of a row-major n x n block.  Returns LAPACK's info.
int potrf_upper( double * U, I32 n )
{
    for( I32 j = 0; j < n; ++j )
    {
        double d = U[static_cast<I64>(j)*n + j];
        for( I32 k = 0; k < j; ++k ) { const double u = U[static_cast<I64>(k)*n + j]; d -= u * u; }
        if( !(d > 0.0) ) { return j + 1; }
        d = std::sqrt( d );
        U[static_cast<I64>(j)*n + j] = d;
        for( I32 c = j + 1; c < n; ++c )
        {
            double s = U[static_cast<I64>(j)*n + c];
            for( I32 k = 0; k < j; ++k ) { s -= U[static_cast<I64>(k)*n + j] * U[static_cast<I64>(k)*n + c]; }
            U[static_cast<I64>(j)*n + c] = s / d;
        }
    }
    return 0;
}

// X <- U^{-T} X for row-major U (n x n upper) and X (n x m, leading dim ld).
void trsm_upper_trans( const double * U, I32 n, double * X, I32 m, I64 ld )
{
    for( I32 r = 0; r < n; ++r )
    {
        double * xr = X + r * ld;
        for( I32 k = 0; k < r; ++k )
        {
            const double u = U[static_cast<I64>(k)*n + r];
            const double * xk = X + k * ld;
            for( I32 c = 0; c < m; ++c ) { xr[c] -= u * xk[c]; }
        }
        const double inv = 1.0 / U[static_cast<I64>(r)*n + r];
        for( I32 c = 0; c < m; ++c ) { xr[c] *= inv; }
    }
}

// X <- U^{-1} X for row-major U (n x n upper) and X (n x m, leading dim ld).
void trsm_upper( const double * U, I32 n, double * X, I32 m, I64 ld )
{
    for( I32 r = n; r-- > 0; )
    {
        double * xr = X + r * ld;
        for( I32 k = r + 1; k < n; ++k )
        {
            const double u = U[static_cast<I64>(r)*n + k];
            const double * xk = X + k * ld;
            for( I32 c = 0; c < m; ++c ) { xr[c] -= u * xk[c]; }
        }
        const double inv = 1.0 / U[static_cast<I64>(r)*n + r];
        for( I32 c = 0; c < m; ++c ) { xr[c] *= inv; }
    }
}

// Multifrontal.hpp:118-504: FetchFromA (:249-321), FetchFromChild
// (:324-436), FactorizeSupernode (:438-475), ComputeUpdateMatrix (:478-504),
// driven in supernode order (children precede parents).
int factor( Oracle & o, const double * values, double reg )
{
    const I32 S = o.sn_count;
    o.aval.resize( o.vperm.size() );
    for( size_t i = 0; i < o.vperm.size(); ++i ) { o.aval[i] = values[o.vperm[i]]; }   // Numeric.hpp:165-180
    o.tri.assign( static_cast<size_t>(o.tri_ptr[S]), 0.0 );                          // Numeric.hpp:256-268
    o.rec.assign( static_cast<size_t>(o.rec_ptr[S]), 0.0 );
    std::vector<std::vector<double>> updates( static_cast<size_t>(S) );
    std::vector<I32> idx( static_cast<size_t>(o.n), 0 );
    bool good = true;

    for( I32 s = 0; s < S; ++s )
    {
        const I32 ib = o.sn_rp[s], ie = o.sn_rp[s+1];
        const I64 jb = o.sn_outer[s], je = o.sn_outer[s+1];
        const I32 n0 = ie - ib, n1 = static_cast<I32>(je - jb);
        double * U0 = &o.tri[o.tri_ptr[s]];
        double * U1 = o.rec.data() + o.rec_ptr[s];
        std::vector<double> & V = updates[s];
        V.assign( static_cast<size_t>(n1) * n1, 0.0 );

        for( I32 i = ib; i < ie; ++i )       // FetchFromA
        {
            const I64 k_end = o.outer[i+1];
            I64 k = o.diag[i];
            U0[static_cast<I64>(n0)*(i-ib) + (o.inner[k]-ib)] = o.aval[k] + reg;
            for( ++k; k < k_end; ++k )
            {
                const I32 j = o.inner[k];
                if( j < ie ) { U0[static_cast<I64>(n0)*(i-ib) + (j-ib)] = o.aval[k]; } else { break; }
            }
            I64 l = jb;
            for( ; k < k_end; ++k )
            {
                const I32 j = o.inner[k];
                while( o.sn_inner[l] < j ) { ++l; }
                U1[static_cast<I64>(n1)*(i-ib) + (l-jb)] = o.aval[k];
            }
        }

        for( I32 i = ib; i < ie; ++i ) { idx[i] = i - ib; }
        for( I64 j = jb; j < je; ++j ) { idx[o.sn_inner[j]] = static_cast<I32>(j - jb); }

        for( I32 c = o.achild_ptr[s]; c < o.achild_ptr[s+1]; ++c )     // FetchFromChild
        {
            const I32 t = o.achild_idx[c];
            const I64 lb = o.sn_outer[t], le = o.sn_outer[t+1];
            const I32 m1 = static_cast<I32>(le - lb);
            const I32 * t_idx = &o.sn_inner[lb];
            const double * W = updates[t].data();
            I32 mid = 0;
            while( mid < m1 && t_idx[mid] < ie ) { ++mid; }
            std::vector<I32> lut( static_cast<size_t>(m1) );
            for( I32 i = 0; i < m1; ++i ) { lut[i] = idx[t_idx[i]]; }
            for( I32 i = 0; i < mid; ++i )
            {
                for( I32 j = i; j < mid; ++j ) { U0[static_cast<I64>(n0)*lut[i] + lut[j]] += W[static_cast<I64>(m1)*i + j]; }
            }
            for( I32 i = 0; i < mid; ++i )
            {
                for( I32 j = mid; j < m1; ++j ) { U1[static_cast<I64>(n1)*lut[i] + lut[j]] += W[static_cast<I64>(m1)*i + j]; }
            }
            for( I32 i = mid; i < m1; ++i )
            {
                for( I32 j = i; j < m1; ++j ) { V[static_cast<I64>(n1)*lut[i] + lut[j]] += W[static_cast<I64>(m1)*i + j]; }
            }
            std::vector<double>().swap( updates[t] );
        }

        if( n0 > 1 )                           // FactorizeSupernode
        {
            good = good && ( potrf_upper( U0, n0 ) == 0 );
            if( n1 > 0 ) { trsm_upper_trans( U0, n0, U1, n1, n1 ); }
        }
        else
        {
            U0[0] = std::sqrt( std::fabs( U0[0] ) );
            const double inv = 1.0 / U0[0];
            for( I32 j = 0; j < n1; ++j ) { U1[j] *= inv; }
        }

        if( n0 > 0 && n1 > 0 )                 // ComputeUpdateMatrix: V -= U1^T U1
        {
            if( n0 > 1 )
            {
                for( I32 i = 0; i < n1; ++i )
                {
                    for( I32 j = i; j < n1; ++j )
                    {
                        double s_ = 0.0;
                        for( I32 k = 0; k < n0; ++k ) { s_ += U1[static_cast<I64>(n1)*k + i] * U1[static_cast<I64>(n1)*k + j]; }
                        V[static_cast<I64>(n1)*i + j] -= s_;
                    }
                }
            }
            else
            {
                for( I32 i = 0; i < n1; ++i )
                {
                    for( I32 j = 0; j < n1; ++j ) { V[static_cast<I64>(n1)*i + j] -= U1[i] * U1[j]; }
                }
            }
        }
    }
    o.good = good;
    return good ? 0 : 1;
}

// LowerSolver.hpp:143-305 (U^T y = b in supernode order) on the permuted,
// row-major n x k block X.
void lower_solve( const Oracle & o, std::vector<double> & X, I32 k )
{
    std::vector<double> X1;
    for( I32 s = 0; s < o.sn_count; ++s )
    {
        const I32 ib = o.sn_rp[s], n0 = o.sn_rp[s+1] - ib;
        const I64 jb = o.sn_outer[s];
        const I32 n1 = static_cast<I32>( o.sn_outer[s+1] - jb );
        const double * U0 = &o.tri[o.tri_ptr[s]];
        const double * U1 = o.rec.data() + o.rec_ptr[s];
        double * X0 = &X[static_cast<I64>(ib) * k];
        trsm_upper_trans( U0, n0, X0, k, k );
        X1.assign( static_cast<size_t>(n1) * k, 0.0 );
        for( I32 r = 0; r < n0; ++r )
        {
            for( I32 j = 0; j < n1; ++j )
            {
                const double u = U1[static_cast<I64>(n1)*r + j];
                for( I32 c = 0; c < k; ++c ) { X1[static_cast<I64>(j)*k + c] -= u * X0[static_cast<I64>(r)*k + c]; }
            }
        }
        for( I32 j = 0; j < n1; ++j )
        {
            double * dst = &X[static_cast<I64>(o.sn_inner[jb+j]) * k];
            for( I32 c = 0; c < k; ++c ) { dst[c] += X1[static_cast<I64>(j)*k + c]; }
        }
    }
}

// UpperSolver.hpp:127-255 (U x = y, parents before children).
void upper_solve( const Oracle & o, std::vector<double> & X, I32 k )
{
    for( I32 s = o.sn_count; s-- > 0; )
    {
        const I32 ib = o.sn_rp[s], n0 = o.sn_rp[s+1] - ib;
        const I64 jb = o.sn_outer[s];
        const I32 n1 = static_cast<I32>( o.sn_outer[s+1] - jb );
        const double * U0 = &o.tri[o.tri_ptr[s]];
        const double * U1 = o.rec.data() + o.rec_ptr[s];
        double * X0 = &X[static_cast<I64>(ib) * k];
        for( I32 r = 0; r < n0; ++r )
        {
            for( I32 j = 0; j < n1; ++j )
            {
                const double u = U1[static_cast<I64>(n1)*r + j];
                const double * xj = &X[static_cast<I64>(o.sn_inner[jb+j]) * k];
                for( I32 c = 0; c < k; ++c ) { X0[static_cast<I64>(r)*k + c] -= u * xj[c]; }
            }
        }
        trsm_upper( U0, n0, X0, k, k );
    }
}

// InputOutput.hpp:8-36 (ReadRightHandSide: X = P B) and :48-78
// (WriteSolution: Y = alpha P^T X + beta Y, where a zero beta leaves the old
// Y unread, Permutation.hpp:380-555).
void run_solve( const Oracle & o, int which, double alpha, const double * B, int ldB,
                double beta, double * Y, int ldY, int nrhs )
{
    const I32 k = std::max( 1, nrhs );
    std::vector<double> X( static_cast<size_t>(o.n) * k );
    for( I32 i = 0; i < o.n; ++i )
    {
        for( I32 c = 0; c < k; ++c ) { X[static_cast<I64>(i)*k + c] = B[static_cast<I64>(ldB) * o.p[i] + c]; }
    }
    if( which != 1 ) { lower_solve( o, X, k ); }
    if( which != 0 ) { upper_solve( o, X, k ); }
    for( I32 i = 0; i < o.n; ++i )
    {
        for( I32 c = 0; c < k; ++c )
        {
            const double x = X[static_cast<I64>(o.pinv[i])*k + c];
            double & y = Y[static_cast<I64>(ldY) * i + c];
            y = (alpha == 0.0 ? 0.0 : alpha * x) + (beta == 0.0 ? 0.0 : beta * y);
        }
    }
}

template<typename T>
void copy_out( const std::vector<T> & v, int64_t * out )
{
    for( size_t i = 0; i < v.size(); ++i ) { out[i] = static_cast<int64_t>(v[i]); }
}

} // namespace

extern "C" {

// CholeskyDecomposition.hpp:313-371 (constructors + Init) followed by
// SymbolicFactorization (Symbolic.hpp:3-66).
void * tb_oracle_analyze( int n, const int64_t * outer, const int32_t * inner,
                          const int32_t * perm, int strategy, int amalgamation_threshold )
{
    Oracle * o = new Oracle();
    o->n = n;
    o->outer.assign( outer, outer + n + 1 );
    o->inner.assign( inner, inner + outer[n] );
    o->p.resize( static_cast<size_t>(n) );
    o->pinv.resize( static_cast<size_t>(n) );
    if( perm != nullptr )
    {
        for( I32 i = 0; i < n; ++i ) { o->p[i] = perm[i]; o->pinv[perm[i]] = i; }
        o->vperm = permute_pattern( o->outer, o->inner, o->p, o->pinv );
    }
    else
    {
        std::iota( o->p.begin(), o->p.end(), 0 );
        std::iota( o->pinv.begin(), o->pinv.end(), 0 );
        o->vperm.resize( o->inner.size() );
        std::iota( o->vperm.begin(), o->vperm.end(), I64(0) );
    }
    require_diag( *o );
    post_ordering( *o );
    find_supernodes( *o, strategy, amalgamation_threshold );
    finish_symbolic( *o );
    return o;
}

void tb_oracle_destroy( void * h ) { delete static_cast<Oracle*>(h); }

int tb_oracle_sn_count( void * h ) { return static_cast<Oracle*>(h)->sn_count; }

int64_t tb_oracle_array_size( void * h, int which )
{
    const Oracle & o = *static_cast<Oracle*>(h);
    switch( which )
    {
        case 0: case 1: return o.n;
        case 2:  return static_cast<int64_t>(o.vperm.size());
        case 3:  return static_cast<int64_t>(o.sn_rp.size());
        case 4:  return static_cast<int64_t>(o.sn_outer.size());
        case 5:  return static_cast<int64_t>(o.sn_inner.size());
        case 6:  return static_cast<int64_t>(o.row_to_sn.size());
        case 7:  return static_cast<int64_t>(o.tri_ptr.size());
        case 8:  return static_cast<int64_t>(o.rec_ptr.size());
        case 9:  return static_cast<int64_t>(o.aparent.size());
        case 10: return static_cast<int64_t>(o.eparent.size());
        case 11: return static_cast<int64_t>(o.outer.size());
        case 12: return static_cast<int64_t>(o.inner.size());
        case 13: return static_cast<int64_t>(o.achild_ptr.size());
        case 14: return static_cast<int64_t>(o.achild_idx.size());
        default: return -1;
    }
}

void tb_oracle_array_copy( void * h, int which, int64_t * out )
{
    const Oracle & o = *static_cast<Oracle*>(h);
    switch( which )
    {
        case 0:  copy_out( o.p, out ); break;
        case 1:  copy_out( o.pinv, out ); break;
        case 2:  copy_out( o.vperm, out ); break;
        case 3:  copy_out( o.sn_rp, out ); break;
        case 4:  copy_out( o.sn_outer, out ); break;
        case 5:  copy_out( o.sn_inner, out ); break;
        case 6:  copy_out( o.row_to_sn, out ); break;
        case 7:  copy_out( o.tri_ptr, out ); break;
        case 8:  copy_out( o.rec_ptr, out ); break;
        case 9:  copy_out( o.aparent, out ); break;
        case 10: copy_out( o.eparent, out ); break;
        case 11: copy_out( o.outer, out ); break;
        case 12: copy_out( o.inner, out ); break;
        case 13: copy_out( o.achild_ptr, out ); break;
        case 14: copy_out( o.achild_idx, out ); break;
        default: break;
    }
}

int tb_oracle_factor( void * h, const double * values, double reg )
{
    return factor( *static_cast<Oracle*>(h), values, reg );
}

int64_t tb_oracle_tri_size( void * h ) { return static_cast<int64_t>(static_cast<Oracle*>(h)->tri.size()); }
int64_t tb_oracle_rec_size( void * h ) { return static_cast<int64_t>(static_cast<Oracle*>(h)->rec.size()); }

void tb_oracle_tri_copy( void * h, double * out )
{
    const auto & v = static_cast<Oracle*>(h)->tri;
    std::copy( v.begin(), v.end(), out );
}

void tb_oracle_rec_copy( void * h, double * out )
{
    const auto & v = static_cast<Oracle*>(h)->rec;
    std::copy( v.begin(), v.end(), out );
}

void tb_oracle_solve( void * h, double alpha, const double * B, int ldB,
                      double beta, double * X, int ldX, int nrhs )
{
    run_solve( *static_cast<Oracle*>(h), 2, alpha, B, ldB, beta, X, ldX, nrhs );
}

void tb_oracle_half_solve( void * h, int which, double alpha, const double * B, int ldB,
                           double beta, double * X, int ldX, int nrhs )
{
    run_solve( *static_cast<Oracle*>(h), which == 0 ? 0 : 1, alpha, B, ldB, beta, X, ldX, nrhs );
}

// InputOutput.hpp:259-297: log det A = 2 * sum log diag(U).
double tb_oracle_log_det( void * h )
{
    const Oracle & o = *static_cast<Oracle*>(h);
    double s = 0.0;
    for( I32 q = 0; q < o.sn_count; ++q )
    {
        const I32 n0 = o.sn_rp[q+1] - o.sn_rp[q];
        for( I32 i = 0; i < n0; ++i ) { s += std::log( o.tri[o.tri_ptr[q] + static_cast<I64>(n0+1)*i] ); }
    }
    return 2.0 * s;
}

} // extern "C"
