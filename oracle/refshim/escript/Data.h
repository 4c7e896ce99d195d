// Stand-in for escript::Data with the accessors the reference assembler uses:
// a coefficient is empty, constant (one data point for all samples) or expanded
// (one data point per quadrature point of every sample).
#pragma once
#include <escript/DataTypes.h>
#include <stdexcept>
namespace escript {
class FunctionSpace {
public:
    int getTypeCode() const { return 0; }
};
class Data {
public:
    Data() {}
    Data(double* p, int dpsize, int perSample, bool expanded)
        : m_p(p), m_dpsize(dpsize), m_perSample(perSample), m_expanded(expanded), m_empty(p == nullptr) {}
    bool isEmpty() const { return m_empty; }
    bool actsExpanded() const { return m_expanded; }
    bool isComplex() const { return false; }
    int getDataPointSize() const { return m_dpsize; }
    void requireWrite() {}
    FunctionSpace getFunctionSpace() const { return FunctionSpace(); }
    const double* getSampleDataRO(DataTypes::index_t s, double) const {
        return m_p + (m_expanded ? (long)s * m_dpsize * m_perSample : 0);
    }
    double* getSampleDataRW(DataTypes::index_t s, double) {
        return m_p + (m_expanded ? (long)s * m_dpsize * m_perSample : 0);
    }
    const DataTypes::cplx_t* getSampleDataRO(DataTypes::index_t, DataTypes::cplx_t) const {
        throw std::runtime_error("complex data not supported by the oracle shim");
    }
    DataTypes::cplx_t* getSampleDataRW(DataTypes::index_t, DataTypes::cplx_t) {
        throw std::runtime_error("complex data not supported by the oracle shim");
    }
private:
    double* m_p = nullptr;
    int m_dpsize = 1;
    int m_perSample = 1;
    bool m_expanded = false;
    bool m_empty = true;
};
}  // namespace escript
