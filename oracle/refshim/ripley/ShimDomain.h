// Stand-in for the parts of ripley::Brick / ripley::Rectangle that the reference
// assemblers call: the element-to-matrix scatter and the face offsets.
#pragma once
#include <escript/AbstractSystemMatrix.h>
#include <ripley/domainhelpers.h>
namespace ripley {
class ShimDomain {
public:
    int dim = 3;
    dim_t m_NN[3] = {0, 0, 0};
    index_t m_faceOffset[6] = {-1, -1, -1, -1, -1, -1};
    dim_t numDOF = 0;
    template <typename Scalar>
    void addToMatrixAndRHS(escript::AbstractSystemMatrix* S, escript::Data& F,
                           const std::vector<Scalar>& EM_S, const std::vector<Scalar>& EM_F,
                           bool addS, bool addF, index_t firstNode, int nEq = 1,
                           int nComp = 1) const;
};
}  // namespace ripley
