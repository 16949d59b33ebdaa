// Host-side symbolic analysis of the supernodal Cholesky factorization.
//
// Produces exactly the symbolic structure of the reference's
// Sparse::CholeskyDecomposition (src/Sparse/CholeskyDecomposition.hpp and
// CholeskyDecomposition/Symbolic.hpp): the postordered permutation, the
// nonzero-value permutation, the supernode partition (SN_rp), the column sets
// of the supernodes' rectangular blocks (SN_outer / SN_inner), row_to_SN, the
// per-supernode value pointers (full n0 x n0 squares and n0 x n1 rectangles)
// and the assembly tree.  The integer outputs are identical to the
// reference's for every input, which the test suite checks against the
// reference's own code.
#pragma once

#include <cstdint>
#include <vector>

namespace tb
{

enum class SupernodeStrategy : int { Maximal = 0, Fundamental = 1, Amalgamated = 2 };

struct SymbolicInput
{
    std::int32_t         n = 0;
    const std::int64_t * outer = nullptr;   // n + 1 row pointers (full symmetric pattern)
    const std::int32_t * inner = nullptr;   // sorted column indices, diagonal present
    const std::int32_t * perm  = nullptr;   // perm[i] = original index at position i; null = identity
    SupernodeStrategy    strategy = SupernodeStrategy::Maximal;
    std::int32_t         amalgamation_threshold = 4;
    std::int32_t         threads = 0;         // host threads of the analysis; <= 0: every hardware thread
};

class Symbolic
{
public:
    // Returns 0 on success or a negative tb status code (invalid pattern,
    // invalid permutation, missing diagonal).
    int analyze( const SymbolicInput & in );

    std::int32_t n = 0;
    std::int64_t nnz = 0;

    // Permutation after postordering: p[i] = original index at position i.
    std::vector<std::int32_t> p, p_inv;
    // Permuted pattern and, per permuted nonzero, its index in the caller's
    // value array.
    std::vector<std::int64_t> outer;
    std::vector<std::int32_t> inner;
    std::vector<std::int64_t> value_perm;
    std::vector<std::int64_t> diag;          // first entry with column >= row

    // Elimination tree of the permuted pattern (roots point to n).
    std::vector<std::int32_t> etree_parent;

    // Supernodes.
    std::int32_t sn_count = 0;
    std::vector<std::int32_t> sn_rp;         // sn_count + 1
    std::vector<std::int64_t> sn_outer;      // sn_count + 1
    std::vector<std::int32_t> sn_inner;      // column indices of the U1 blocks
    std::vector<std::int32_t> row_to_sn;     // n
    std::vector<std::int64_t> sn_tri_ptr;    // sn_count + 1, prefix sums of n0^2
    std::vector<std::int64_t> sn_rec_ptr;    // sn_count + 1, prefix sums of n0*n1
    std::int32_t max_n0 = 0, max_n1 = 0;

    // Assembly tree over supernodes; the virtual root is sn_count.
    std::vector<std::int32_t> atree_parent;  // sn_count
    std::vector<std::int32_t> atree_child_ptr, atree_child_idx;

    std::int32_t n0( std::int32_t s ) const { return sn_rp[s+1] - sn_rp[s]; }
    std::int32_t n1( std::int32_t s ) const { return static_cast<std::int32_t>( sn_outer[s+1] - sn_outer[s] ); }

private:
    std::int32_t threads_ = 0;

    struct Forest
    {
        std::vector<std::int32_t> child_ptr, child_idx, desc;
        std::vector<std::int32_t> postorder;
    };

    void permute_pattern( const std::vector<std::int32_t> & rows, const std::vector<std::int32_t> & cols_inv,
                          std::vector<std::int64_t> & moved_from );
    void locate_diagonal();
    void elimination_tree();
    static void forest_of( const std::vector<std::int32_t> & parent, Forest & f, bool with_order );
    static bool postordered( const std::vector<std::int32_t> & parent, const std::vector<std::int32_t> & desc );
    void supernode_starts( const Forest & et, std::vector<std::uint8_t> & fresh ) const;
    void supernodes( SupernodeStrategy strategy, std::int32_t threshold, const Forest & et );
    void assembly_tree();
};

} // namespace tb
