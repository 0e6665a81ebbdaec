"""Flat random-forest format for the GPU classifier.

The reference classifies each (pixel, d) feature vector with a scikit-learn
RandomForestClassifier (trained at train.py:287-289, applied with
predict_proba at test.py:620).  sklearn walks each tree with
`float32(x[f]) <= threshold` (threshold in float64; sklearn/tree/_tree.pyx,
Tree._apply_dense) and averages the leaves' class fractions over the trees in
float64 (sklearn/ensemble/_forest.py, ForestClassifier.predict_proba).

FlatForest keeps those trees as flat arrays (sklearn's own node numbering,
per-tree offsets) and is what both the GPU packer and the tests use:

  roots[t]       first node of tree t in the flat arrays
  feature[n]     split feature (-2 on leaves, as sklearn)
  threshold[n]   split threshold, float64 (sklearn's)
  left/right[n]  children, tree-local indices; -1 on leaves
  value0[n]      class-0 fraction of the node's training samples, float64
                 (class 0 = wrong match, so P0 is the matching cost the
                 reference feeds to its post-processing, test.py:144-145)
  value1[n]      class-1 fraction (sklearn keeps both; 1 - value0 is not
                 always bit-equal to it)

pack() turns it into the device layout (see csrc/rf.cu): per tree, nodes
renumbered breadth-first so that the two children of a node are adjacent, and
each 8-byte node holds a float32 threshold t32 = the largest float32 <= the
float64 threshold (for a float32 x, x <= thr64 exactly when x <= t32) and a
32-bit word: bit 31 leaf flag; bits 0-4 feature; bits 5-30 index of the left
child (the right child follows it).  A leaf's word holds the index of its
float64 (class-0, class-1) fractions in the leaf-value array.
"""
import numpy as np

LEAF_FLAG = np.uint32(1 << 31)


class FlatForest:
    def __init__(self, roots, feature, threshold, left, right, value0, n_features=20, value1=None):
        self.roots = np.ascontiguousarray(roots, np.int32)
        self.feature = np.ascontiguousarray(feature, np.int32)
        self.threshold = np.ascontiguousarray(threshold, np.float64)
        self.left = np.ascontiguousarray(left, np.int32)
        self.right = np.ascontiguousarray(right, np.int32)
        self.value0 = np.ascontiguousarray(value0, np.float64)
        self.value1 = np.ascontiguousarray(1.0 - self.value0 if value1 is None else value1, np.float64)
        self.n_features = int(n_features)

    @property
    def n_trees(self):
        return int(self.roots.shape[0])

    @property
    def n_nodes(self):
        return int(self.feature.shape[0])

    def tree_sizes(self):
        ends = np.append(self.roots[1:], self.n_nodes)
        return ends - self.roots

    @classmethod
    def from_sklearn(cls, rf):
        """Flatten a fitted binary RandomForestClassifier (classes [0, 1])."""
        classes = list(np.asarray(rf.classes_).tolist())
        if len(classes) != 2:
            raise ValueError("expected a binary classifier, got classes %r" % (classes,))
        roots, feat, thr, lft, rgt, val, val1 = [], [], [], [], [], [], []
        off = 0
        for est in rf.estimators_:
            t = est.tree_
            roots.append(off)
            feat.append(t.feature.astype(np.int32))
            thr.append(t.threshold.astype(np.float64))
            lft.append(t.children_left.astype(np.int32))
            rgt.append(t.children_right.astype(np.int32))
            v = t.value[:, 0, :].astype(np.float64)
            s = v.sum(axis=1)
            # sklearn >= 1.4 stores fractions; older versions store counts.
            norm = np.abs(s - 1.0) < 1e-9
            den = np.where(s > 0, s, 1.0)
            val.append(np.where(norm, v[:, 0], v[:, 0] / den))
            val1.append(np.where(norm, v[:, 1], v[:, 1] / den))
            off += t.node_count
        return cls(np.array(roots), np.concatenate(feat), np.concatenate(thr), np.concatenate(lft),
                   np.concatenate(rgt), np.concatenate(val), n_features=rf.n_features_in_,
                   value1=np.concatenate(val1))

    def save(self, path):
        np.savez_compressed(path, roots=self.roots, feature=self.feature, threshold=self.threshold,
                            left=self.left, right=self.right, value0=self.value0,
                            value1=self.value1, n_features=np.int32(self.n_features))

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z["roots"], z["feature"], z["threshold"], z["left"], z["right"], z["value0"],
                   int(z["n_features"]), z["value1"] if "value1" in z.files else None)

    def pack(self):
        """Device layout: nodes uint32 [M,2], leaf_values float64 [K,2],
        tree_offsets int32 [T+1], and orig int32 [M] (each packed node's
        sklearn node id within its tree)."""
        if self.n_features > 32:
            raise ValueError("the packed node has 5 feature bits")
        nodes_out, leafv, offs, origs = [], [], [0], []
        total = 0
        nleaf = 0
        for t in range(self.n_trees):
            base = int(self.roots[t])
            end = int(self.roots[t + 1]) if t + 1 < self.n_trees else self.n_nodes
            lft = self.left[base:end]
            rgt = self.right[base:end]
            # breadth-first renumbering, children adjacent
            order = np.empty(end - base, np.int64)
            order[0] = 0
            head, tail = 0, 1
            while head < tail:
                n = order[head]
                head += 1
                if lft[n] >= 0:
                    order[tail] = lft[n]
                    order[tail + 1] = rgt[n]
                    tail += 2
            order = order[:tail]
            newidx = np.empty(end - base, np.int64)
            newidx[order] = np.arange(tail)
            g = base + order
            is_leaf = self.left[g] < 0
            th = self.threshold[g]
            t32 = th.astype(np.float32)
            over = t32.astype(np.float64) > th
            t32[over] = np.nextafter(t32[over], np.float32(-np.inf))
            t32[is_leaf] = 0.0
            word = np.zeros(tail, np.uint32)
            nl = int(is_leaf.sum())
            word[is_leaf] = LEAF_FLAG | (np.arange(nleaf, nleaf + nl, dtype=np.uint32))
            inner = ~is_leaf
            child = total + newidx[self.left[g[inner]]]
            if tail and child.size and child.max() >= (1 << 26):
                raise ValueError("forest too large for the 26-bit child index")
            word[inner] = (self.feature[g[inner]].astype(np.uint32)
                           | (child.astype(np.uint32) << np.uint32(5)))
            lv = np.stack([self.value0[g[is_leaf]], self.value1[g[is_leaf]]], axis=1)
            nodes = np.empty((tail, 2), np.uint32)
            nodes[:, 0] = t32.view(np.uint32)
            nodes[:, 1] = word
            nodes_out.append(nodes)
            leafv.append(lv)
            origs.append(order.astype(np.int32))
            nleaf += nl
            total += tail
            offs.append(total)
        return (np.ascontiguousarray(np.concatenate(nodes_out)),
                np.ascontiguousarray(np.concatenate(leafv)), np.asarray(offs, np.int32),
                np.concatenate(origs))
