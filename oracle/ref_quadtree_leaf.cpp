// Compiles the reference's quadtree.cpp, unmodified and from where it lies,
// with its leaf-size macro MAX_LEAF_DOFS (a plain #define of 32 in
// kern_interp/quadtree/quadtree.h:10) bound to a runtime variable, so one
// reference build serves the 32-dof default and the 64-point leaves of the
// benchmark workloads.  Test infrastructure only.
#include "kern_interp/quadtree/quadtree.h"
#undef MAX_LEAF_DOFS
extern int kiref_max_leaf_dofs;
#define MAX_LEAF_DOFS kiref_max_leaf_dofs
#include "kern_interp/quadtree/quadtree.cpp"

int kiref_max_leaf_dofs = 32;
