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

pack() turns it into the device layout (csrc/rf.cu): every tree cut into
two-level blocks of 32 bytes -- one DRAM/L2 sector -- so one load serves two
levels of a walk:
  words 0-2  float32 thresholds of the block's root (node 0) and of its two
             children (nodes 1, 2); each is t32 = the largest float32 <= the
             float64 threshold (for a float32 x, x <= thr64 exactly when
             x <= t32)
  word 3     features of nodes 0, 1, 2 in bytes 0, 1, 2 (0xFF: a leaf)
  words 4-7  the four grandchildren: node 1's left/right, node 2's left/right;
             bit 31 set = leaf index, clear = index of the block rooted there.
A leaf at node 0 keeps its leaf index in word 4, a leaf at node 1 in word 4,
a leaf at node 2 in word 6.  Blocks are numbered breadth-first per tree, so
the top blocks of every tree form a prefix that can be staged in shared
memory.  Leaf values are float64 (class-0, class-1) fractions.
"""
import numpy as np

LEAF_FLAG = np.uint32(1 << 31)
LEAF_FEATURE = 0xFF


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

    def node_depths(self):
        """Depth of every node (root 0), indexed like `feature`: the number of
        comparisons a walk makes before it stands on that node."""
        depth = np.zeros(self.n_nodes, np.int32)
        for t in range(self.n_trees):
            base = int(self.roots[t])
            stack = [0]
            while stack:
                n = stack.pop()
                if self.left[base + n] >= 0:
                    for c in (int(self.left[base + n]), int(self.right[base + n])):
                        depth[base + c] = depth[base + n] + 1
                        stack.append(c)
        return depth

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
        """Device layout (see the module docstring): blocks uint32 [NB, 8],
        leaf values float64 [K, 2], per-tree block offsets int32 [T+1], and
        leaf_node int32 [K] (each leaf's sklearn node id within its tree)."""
        if self.n_features >= LEAF_FEATURE:
            raise ValueError("features must be numbered below %d" % LEAF_FEATURE)
        blocks, leafv, offs, leaf_node = [], [], [0], []
        nb_total = 0
        for t in range(self.n_trees):
            base = int(self.roots[t])
            lft, rgt = self.left, self.right

            def leaf_id(n):
                leafv.append((self.value0[base + n], self.value1[base + n]))
                leaf_node.append(n)
                return len(leafv) - 1

            def t32(n):
                th = self.threshold[base + n]
                v = np.float32(th)
                if np.float64(v) > th:
                    v = np.nextafter(v, np.float32(-np.inf))
                return v

            tree_blocks = []
            queue = [0]  # block roots, breadth-first
            qi = 0
            while qi < len(queue):
                r = queue[qi]
                qi += 1
                thr = np.zeros(3, np.float32)
                feat = [LEAF_FEATURE] * 3
                child = [0, 0, 0, 0]
                pending = []  # (slot, node) whose block index is assigned below
                if lft[base + r] < 0:
                    child[0] = leaf_id(r)
                else:
                    thr[0] = t32(r)
                    feat[0] = int(self.feature[base + r])
                    for k, n in ((1, int(lft[base + r])), (2, int(rgt[base + r]))):
                        slot = 2 * (k - 1)
                        if lft[base + n] < 0:
                            child[slot] = leaf_id(n)
                        else:
                            thr[k] = t32(n)
                            feat[k] = int(self.feature[base + n])
                            for j, c in enumerate((int(lft[base + n]), int(rgt[base + n]))):
                                if lft[base + c] < 0:
                                    child[slot + j] = int(LEAF_FLAG) | leaf_id(c)
                                else:
                                    pending.append((slot + j, c))
                for slot, c in pending:
                    child[slot] = nb_total + len(queue)
                    queue.append(c)
                row = np.zeros(8, np.uint32)
                row[0:3] = thr.view(np.uint32)
                row[3] = feat[0] | (feat[1] << 8) | (feat[2] << 16)
                row[4:8] = child
                tree_blocks.append(row)
            blocks.extend(tree_blocks)
            nb_total += len(tree_blocks)
            offs.append(nb_total)
        if nb_total >= int(LEAF_FLAG) or len(leafv) >= int(LEAF_FLAG):
            raise ValueError("forest too large for 31-bit block / leaf indices")
        return (np.ascontiguousarray(np.stack(blocks)), np.asarray(leafv, np.float64),
                np.asarray(offs, np.int32), np.asarray(leaf_node, np.int32))
