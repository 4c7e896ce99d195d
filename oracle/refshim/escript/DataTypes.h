// Minimal stand-in for escript's DataTypes.h: just the scalar and index types the
// reference's ripley assembler and paso solver sources name.  Used only to compile
// those reference sources in place for the oracle (oracle/build_ref.sh).
#pragma once
#include <complex>
#include <limits>
#include <vector>
namespace escript {
namespace DataTypes {
typedef double real_t;
typedef std::complex<double> cplx_t;
typedef int index_t;
typedef index_t dim_t;
inline real_t real_t_eps() { return std::numeric_limits<real_t>::epsilon(); }
}  // namespace DataTypes
}  // namespace escript
