"""Rebuild a scikit-learn RandomForestClassifier from a FlatForest (test and
baseline infrastructure only).

The reference runs sklearn's own predict_proba (test.py:603-620).  The forest
fixture is stored flat (cbmv_b200.forest.FlatForest); to time and check the
reference path with sklearn itself, the trees are put back into sklearn Tree
objects through Tree.__setstate__ (sklearn/tree/_tree.pyx), with the split
fields and class fractions of the stored forest.  Fields that prediction does
not read (impurity, sample counts) are filled with neutral values.
"""
import numpy as np


def to_sklearn(flat, n_jobs=1):
    from sklearn.ensemble import RandomForestClassifier
    from sklearn.tree import DecisionTreeClassifier
    from sklearn.tree._tree import NODE_DTYPE, Tree

    classes = np.array([0.0, 1.0])
    n_classes = np.array([2], dtype=np.intp)
    ests = []
    ends = np.append(flat.roots[1:], flat.n_nodes)
    for t in range(flat.n_trees):
        a, b = int(flat.roots[t]), int(ends[t])
        m = b - a
        nodes = np.zeros(m, dtype=NODE_DTYPE)
        nodes["left_child"] = flat.left[a:b]
        nodes["right_child"] = flat.right[a:b]
        nodes["feature"] = flat.feature[a:b]
        nodes["threshold"] = flat.threshold[a:b]
        nodes["n_node_samples"] = 1
        nodes["weighted_n_node_samples"] = 1.0
        values = np.stack([flat.value0[a:b], flat.value1[a:b]], axis=1)[:, None, :].astype(np.float64)
        depth = _depth(flat.left[a:b], flat.right[a:b])
        tree = Tree(flat.n_features, n_classes, 1)
        tree.__setstate__({"max_depth": depth, "node_count": m, "nodes": nodes,
                           "values": np.ascontiguousarray(values)})
        est = DecisionTreeClassifier()
        est.tree_ = tree
        est.n_features_in_ = flat.n_features
        est.n_outputs_ = 1
        est.classes_ = classes
        est.n_classes_ = 2
        est.max_features_ = flat.n_features
        ests.append(est)
    rf = RandomForestClassifier(n_estimators=flat.n_trees, n_jobs=n_jobs)
    rf.estimators_ = ests
    rf.classes_ = classes
    rf.n_classes_ = 2
    rf.n_outputs_ = 1
    rf.n_features_in_ = flat.n_features
    rf.estimator_ = DecisionTreeClassifier()
    return rf


def _depth(left, right):
    depth = np.zeros(left.shape[0], np.int64)
    for n in range(left.shape[0]):  # sklearn numbers children after parents
        if left[n] >= 0:
            depth[left[n]] = depth[n] + 1
            depth[right[n]] = depth[n] + 1
    return int(depth.max())
