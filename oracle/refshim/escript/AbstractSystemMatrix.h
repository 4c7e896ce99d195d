// Stand-in for escript::AbstractSystemMatrix: a CSR matrix view the shim domain
// scatters element matrices into (see ref_driver.cpp).
#pragma once
namespace escript {
class AbstractSystemMatrix {
public:
    virtual ~AbstractSystemMatrix() {}
    int getRowBlockSize() const { return nb; }
    int getColumnBlockSize() const { return nb; }
    int nb = 1;  // block size (numEq = numComp) of a PDE system
    const int* ptr = nullptr;
    const int* idx = nullptr;
    double* val = nullptr;
    long n = 0;
};
}  // namespace escript
