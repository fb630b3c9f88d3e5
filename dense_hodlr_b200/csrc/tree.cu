// The HODLR tree as level arrays: createDefaultTree (src/HODLR_Tree.cpp:33-132)
// and userTree_To_HODLRTree (src/HODLR_Tree.cpp:207-327).
#include "handle.h"

namespace hodlr_impl {

void push_inner_node(hodlr_t h, int level, int mn, int split, int mx, int u) {
  if ((int)h->lv.size() <= level) h->lv.resize(level + 1);
  Level& L = h->lv[level];
  L.nmin.push_back(mn);
  L.nsplit.push_back(split);
  L.nmax.push_back(mx);
  const bool b = u >= 0 && !h->ut_tmin.empty();
  L.tmin.push_back(b ? h->ut_tmin[u] : -1);
  L.bmin.push_back(b ? h->ut_bmin[u] : -1);
  L.tmax.push_back(b ? h->ut_tmax[u] : -1);
  L.bmax.push_back(b ? h->ut_bmax[u] : -1);
}

// createDefaultTree (src/HODLR_Tree.cpp:33-132): root is a leaf iff N < leaf;
// a child splits iff its size > leaf; a left-type child splits at
// min + floor(s/2) - 1, a right-type child at max - floor(s/2).  Nodes of a
// level are listed left to right (pre-order pushes), leaves in index order.
// The tree of one system on points [o, o + N): inner nodes appended level by
// level (pre-order, left before right), leaves in index order.
void build_subtree(hodlr_t h, int o, int N) {
  const int leaf = h->leaf;
  if (N < leaf || N < 2) {
    h->leaf_min.push_back(o);
    h->leaf_size.push_back(N);
    return;
  }
  struct Fr {
    int level, mn, split, mx;
  };
  std::vector<Fr> stack;
  stack.push_back({0, o, o + N / 2 - 1, o + N - 1});
  auto push_inner = [&](const Fr& f) { push_inner_node(h, f.level, f.mn, f.split, f.mx); };
  // explicit pre-order, left before right
  while (!stack.empty()) {
    Fr f = stack.back();
    stack.pop_back();
    push_inner(f);
    int top = f.split - f.mn + 1, bott = f.mx - f.split;
    Fr right{f.level + 1, f.mn + top, -1, f.mx};
    Fr left{f.level + 1, f.mn, -1, f.mn + top - 1};
    bool rsplit = bott > leaf, lsplit = top > leaf;
    if (rsplit) right.split = f.mx - bott / 2;
    if (lsplit) left.split = f.mn + top / 2 - 1;
    if (rsplit) stack.push_back(right);
    if (lsplit) stack.push_back(left);
  }
  // Walk the tree again to list the leaves in index order.
  std::vector<Fr> st2;
  st2.push_back({0, o, o + N / 2 - 1, o + N - 1});
  while (!st2.empty()) {
    Fr f = st2.back();
    st2.pop_back();
    if (f.split < 0) {
      h->leaf_min.push_back(f.mn);
      h->leaf_size.push_back(f.mx - f.mn + 1);
      continue;
    }
    int top = f.split - f.mn + 1, bott = f.mx - f.split;
    Fr right{f.level + 1, f.mn + top, -1, f.mx};
    Fr left{f.level + 1, f.mn, -1, f.mn + top - 1};
    if (bott > leaf) right.split = f.mx - bott / 2;
    if (top > leaf) left.split = f.mn + top / 2 - 1;
    st2.push_back(right);
    st2.push_back(left);
  }
}

// ---- user index trees (userTree_To_HODLRTree, src/HODLR_Tree.cpp:207-327)

// An inner node with a given split and the default rules below it
// (createDefaultTree from that node): a child splits iff its size exceeds the
// leaf size, the left-type child with floor(s/2) rows on top, the right-type
// child with ceil(s/2).
void grow_default(hodlr_t h, int level, int mn, int split, int mx) {
  push_inner_node(h, level, mn, split, mx);
  const int top = split - mn + 1, bott = mx - split;
  if (top > h->leaf) {
    grow_default(h, level + 1, mn, mn + top / 2 - 1, split);
  } else {
    h->leaf_min.push_back(mn);
    h->leaf_size.push_back(top);
  }
  if (bott > h->leaf) {
    grow_default(h, level + 1, split + 1, mx - bott / 2, mx);
  } else {
    h->leaf_min.push_back(split + 1);
    h->leaf_size.push_back(bott);
  }
}

// Node [mn, mx] of user node u: a leaf when it is no larger than the leaf size
// and has no split; otherwise split where u says, with u's children, or, if
// u has none, default children (the right one with floor(s/2) rows on top,
// as the reference builds them).  Returns false for an invalid user tree.
bool user_subtree(hodlr_t h, int level, int mn, int mx, int u, std::vector<char>& seen) {
  if (u < 0 || u >= (int)h->ut_split.size() || seen[u]) return false;
  seen[u] = 1;
  const int size = mx - mn + 1, sp = h->ut_split[u];
  if (size <= h->leaf && sp == -1) {
    h->leaf_min.push_back(mn);
    h->leaf_size.push_back(size);
    return true;
  }
  if (sp < mn || sp >= mx) return false;
  push_inner_node(h, level, mn, sp, mx, u);
  const int l = h->ut_left[u], r = h->ut_right[u];
  if (l < 0 && r < 0) {
    const int ls = sp - mn + 1, rs = mx - sp;
    if (ls > h->leaf) {
      grow_default(h, level + 1, mn, mn + ls / 2 - 1, sp);
    } else {
      h->leaf_min.push_back(mn);
      h->leaf_size.push_back(ls);
    }
    if (rs > h->leaf) {
      grow_default(h, level + 1, sp + 1, sp + rs / 2, mx);
    } else {
      h->leaf_min.push_back(sp + 1);
      h->leaf_size.push_back(rs);
    }
    return true;
  }
  if (l < 0 || r < 0) return false;
  return user_subtree(h, level + 1, mn, sp, l, seen) &&
         user_subtree(h, level + 1, sp + 1, mx, r, seen);
}

// One tree, or a forest: every system's root sits at level 0, so a level's
// blocks (and its ACA launch, its batched leaf LUs and GEMMs) span all
// systems.
void build_tree(hodlr_t h) {
  h->lv.clear();
  h->leaf_min.clear();
  h->leaf_size.clear();
  if (h->nsys == 0 && !h->ut_split.empty()) {
    std::vector<char> seen(h->ut_split.size(), 0);
    if (!user_subtree(h, 0, 0, h->n - 1, 0, seen)) {  // invalid: the caller restores
      h->lv.clear();
      h->leaf_min.clear();
      h->leaf_size.clear();
      return;
    }
  } else if (h->nsys == 0)
    build_subtree(h, 0, h->n);
  else
    for (int q = 0; q < h->nsys; ++q)
      build_subtree(h, h->sys_off[q], h->sys_off[q + 1] - h->sys_off[q]);
  for (auto& L : h->lv) {
    L.ub_max = 0;
    for (int q = 0; q < L.nblocks(); ++q) {
      int r0, c0, m, n;
      block_geom(L, q, r0, c0, m, n);
      L.ub_max = std::max(L.ub_max, std::min(m, n));
    }
  }
  h->smax = 0;
  for (int s : h->leaf_size) h->smax = std::max(h->smax, s);
}

}  // namespace hodlr_impl
