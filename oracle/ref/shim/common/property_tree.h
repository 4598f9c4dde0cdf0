/* Build shim for compiling HiFlow3's lmp CPU sources outside their CMake
 * build (test infrastructure only).
 *
 * HiFlow3's real common/property_tree.h wraps tinyxml2 and MPI broadcast;
 * neither library is present here.  Within the lmp CPU sources only
 * read_LA_parameters (lmp/init_vec_mat.cc:51) reads a PropertyTree, and the
 * oracle never calls it, so every lookup returns the caller's default. */
#ifndef B200LA_ORACLE_SHIM_PROPERTY_TREE_H
#define B200LA_ORACLE_SHIM_PROPERTY_TREE_H

#include <string>

namespace hiflow {

class PropertyTree {
public:
  PropertyTree() {}
  bool contains(const std::string &) const { return false; }
  PropertyTree const &operator[](const std::string &) const { return *this; }
  template < typename T > T get() const { return T(); }
  template < typename T > T get(T def) const { return def; }
};

} // namespace hiflow

#endif
