// Stand-in declaration of ripley::DefaultAssembler2D with the member functions the
// reference DefaultAssembler2D.cpp defines, bound to the shim domain.
#pragma once
#include <escript/AbstractSystemMatrix.h>
#include <escript/Data.h>
#include <ripley/ShimDomain.h>
#include <ripley/domainhelpers.h>
#include <algorithm>
#include <vector>
namespace ripley {
template <class Scalar = double>
class DefaultAssembler2D {
public:
    DefaultAssembler2D(const ShimDomain* dom, const double* dx, const dim_t* NE, const dim_t* NN)
        : domain(dom), m_dx(dx), m_NE(NE), m_NN(NN) {}
    virtual ~DefaultAssembler2D() {}
#define RIPLEY_SHIM_FULL(name) virtual void name(escript::AbstractSystemMatrix* mat, escript::Data& rhs, \
        const escript::Data& A, const escript::Data& B, const escript::Data& C, \
        const escript::Data& D, const escript::Data& X, const escript::Data& Y) const;
#define RIPLEY_SHIM_BND(name) virtual void name(escript::AbstractSystemMatrix* mat, escript::Data& rhs, \
        const escript::Data& d, const escript::Data& y) const;
#define RIPLEY_SHIM_MAP(name) virtual void name(escript::AbstractSystemMatrix* mat, escript::Data& rhs, \
        const DataMap& coefs) const;
    RIPLEY_SHIM_FULL(assemblePDESingle)
    RIPLEY_SHIM_BND(assemblePDEBoundarySingle)
    RIPLEY_SHIM_FULL(assemblePDESingleReduced)
    RIPLEY_SHIM_BND(assemblePDEBoundarySingleReduced)
    RIPLEY_SHIM_FULL(assemblePDESystem)
    RIPLEY_SHIM_BND(assemblePDEBoundarySystem)
    RIPLEY_SHIM_FULL(assemblePDESystemReduced)
    RIPLEY_SHIM_BND(assemblePDEBoundarySystemReduced)
    RIPLEY_SHIM_MAP(assemblePDESingle)
    RIPLEY_SHIM_MAP(assemblePDEBoundarySingle)
    RIPLEY_SHIM_MAP(assemblePDESingleReduced)
    RIPLEY_SHIM_MAP(assemblePDEBoundarySingleReduced)
    RIPLEY_SHIM_MAP(assemblePDESystem)
    RIPLEY_SHIM_MAP(assemblePDEBoundarySystem)
    RIPLEY_SHIM_MAP(assemblePDESystemReduced)
    RIPLEY_SHIM_MAP(assemblePDEBoundarySystemReduced)
#undef RIPLEY_SHIM_FULL
#undef RIPLEY_SHIM_BND
#undef RIPLEY_SHIM_MAP
    void collateFunctionSpaceTypes(std::vector<int>& fsTypes, const DataMap& coefs) const;
protected:
    const ShimDomain* domain;
    const double* m_dx;
    const dim_t* m_NE;
    const dim_t* m_NN;
};
}  // namespace ripley
