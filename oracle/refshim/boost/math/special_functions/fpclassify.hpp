// Stand-in for boost::math::isnan, the only boost facility paso's Solver.cpp uses.
#pragma once
#include <cmath>
namespace boost { namespace math { using std::isnan; } }
