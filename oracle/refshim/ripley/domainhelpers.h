// Stand-in for ripley/domainhelpers.h: the coefficient map type and lookups.
#pragma once
#include <escript/Data.h>
#include <map>
#include <string>
#include <vector>
namespace ripley {
typedef escript::DataTypes::index_t index_t;
typedef escript::DataTypes::dim_t dim_t;
typedef escript::DataTypes::real_t real_t;
typedef escript::DataTypes::cplx_t cplx_t;
typedef std::vector<index_t> IndexVector;
typedef std::map<std::string, escript::Data> DataMap;
inline const escript::Data unpackData(const std::string& key, const DataMap& m) {
    DataMap::const_iterator i = m.find(key);
    return i == m.end() ? escript::Data() : i->second;
}
inline bool isNotEmpty(const std::string& key, const DataMap& m) {
    DataMap::const_iterator i = m.find(key);
    return i != m.end() && !i->second.isEmpty();
}
}  // namespace ripley
