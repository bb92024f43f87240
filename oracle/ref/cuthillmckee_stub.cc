// Test-infrastructure stub that stands in for the reference's
// Solver/cuthillmckee.cc, which needs METIS (cuthillmckee.cc:26, calls at
// :126-135). METIS is not vendored and no version is pinned. The Cuthill-McKee
// ordering only permutes the block-ILU smoother (Solver/stdsolver.cc:1600-1625);
// the oracle configurations use the Jacobi and Vanka smoothers, and PermutateIlu
// skips the ordering for Vanka (stdsolver.cc:1607), so this stub keeps the
// identity permutation and is never reached on the hot path.
#include "cuthillmckee.h"

namespace Gascoigne {

CuthillMcKee::CuthillMcKee(const StencilInterface* s)
  : S(s)
  , CS(nullptr)
  , DS(nullptr)
{}

CuthillMcKee::CuthillMcKee()
  : S(nullptr)
  , CS(nullptr)
  , DS(nullptr)
{}

void
CuthillMcKee::Permutate(IntVector& perm)
{
  for (size_t i = 0; i < perm.size(); ++i)
    perm[i] = static_cast<int>(i);
}

} // namespace Gascoigne
