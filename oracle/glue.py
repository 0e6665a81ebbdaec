"""Python-3 restatement of the reference's Python-2 drivers (test infrastructure only).

The reference's test.py / train.py cannot run here (Python 2: print
statements, cPickle, scipy.misc.imread).  These functions restate the ~150
lines of glue on the cost-volume path, line for line, over any backend that
exposes the reference's module surface: oracle.ref (the reference's own
compiled code), oracle.cpu (the C restatement) or cbmv_b200's drop-in shims.
"""
import math

import numpy as np

# Testing.__init__ defaults, test.py:44-73
PARAMS = dict(censw=11, nccw=3, sadw=5, pi1=1.3, pi2=10, sgm_q1=2.2, sgm_q2=3, alpha1=1.4,
              tau_so=.12, sgm_i=2, L1=6, tau1=.07, cbca_i1=0, cbca_i2=4, median_i=1,
              median_w=3, blur_sigma=2.2, blur_t=1.3)
CENS_SIGMA = 2 * 8 ** 2   # test.py:71
NCC_SIGMA = 0.02          # test.py:72
SAD_SIGMA = 2 * 100 ** 2  # test.py:73
TEST_BATCH = 100000       # test.py:55


def gaussian(sigma):
    """Testing.__gaussian, test.py:108-118 (centre offset by one, as written)."""
    kr = math.ceil(sigma * 3)
    ks = int(kr * 2 + 1)
    k = np.zeros((ks, ks))
    for i in range(0, ks):
        for j in range(0, ks):
            y = (i - 1) - kr
            x = (j - 1) - kr
            k[i, j] = math.exp(-(x * x + y * y) / (2 * sigma * sigma))
    return k.astype(np.float32)


def get_costs(mtc, fte, iml, imr, d, censw=11, nccw=3, sadw=5):
    """Testing.__get_costs, test.py:122-138.  All four volumes [H,W,D] f64."""
    costcensus = mtc.census(iml, imr, d, censw).astype(np.float64)
    costncc = mtc.nccNister(iml, imr, d, nccw)
    costncc = fte.swap_axes(costncc)
    sobl = mtc.sobel(iml)
    sobr = mtc.sobel(imr)
    costsob = mtc.sadsob(sobl, sobr, d, 5).astype(np.float64)
    costsob = fte.swap_axes(costsob)
    costsad = mtc.zsad(iml, imr, d, sadw).astype(np.float64)
    costsad = fte.swap_axes(costsad)
    return costcensus, costncc, costsob, costsad


def extract_features_lr(fte, census, ncc, sobel, sad):
    """Testing.__extract_features_lr, test.py:521-595: [rows*W*D, 20] f64."""
    dims = census.shape
    n = dims[0] * dims[1] * dims[2]
    vols = []
    for v in (census, ncc, sobel, sad):
        vr = fte.get_right_cost(v)
        vols.append((np.reshape(v, [dims[0] * dims[1], dims[2]]),
                     np.reshape(vr, [dims[0] * dims[1], dims[2]])))
    features = np.empty((n, 20))
    for k, (v, _) in enumerate(vols):
        features[:, k] = np.reshape(v, [n])
    es = (.01, 1.01, .01, .01)
    sig = (CENS_SIGMA, NCC_SIGMA, SAD_SIGMA, SAD_SIGMA)
    for k, (v, _) in enumerate(vols):
        features[:, 4 + k] = np.reshape(fte.extract_ratio(v, es[k]), [n])
    for k, (v, _) in enumerate(vols):
        features[:, 8 + k] = np.reshape(fte.extract_likelihood(v, sig[k]), [n])
    for k, (_, vr) in enumerate(vols):
        r_pkrn = np.reshape(fte.extract_ratio(vr, es[k]), [dims[0], dims[1], dims[2]])
        features[:, 12 + k] = np.reshape(fte.get_left_cost(r_pkrn), [n])
        r_aml = np.reshape(fte.extract_likelihood(vr, sig[k]), [dims[0], dims[1], dims[2]])
        features[:, 16 + k] = np.reshape(fte.get_left_cost(r_aml), [n])
    return features


def test_model(mtc, fte, predict_proba, iml, imr, d, batch=TEST_BATCH, rows=None):
    """Testing.test_model, test.py:597-626.

    predict_proba(features) -> [N,2] (sklearn's RandomForestClassifier in the
    reference).  `rows` limits the pass to the first `rows` image rows (a
    bounded sample of the workload; None = all rows).  The reference's
    np.append accumulation is kept as written."""
    census, ncc, sobel, sad = get_costs(mtc, fte, iml, imr, d)
    h, w = iml.shape
    hh = h if rows is None else min(h, rows)
    proba = np.empty((0, 2))
    r_s = int(math.floor(batch / w))
    batch_index = 0
    while batch_index < hh:
        e = min(batch_index + r_s, hh)
        features = extract_features_lr(fte, census[batch_index:e, :, :], ncc[batch_index:e, :, :],
                                       sobel[batch_index:e, :, :], sad[batch_index:e, :, :])
        batch_proba = predict_proba(features)
        batch_index += r_s
        proba = np.append(proba, batch_proba, axis=0)
    return proba


def normalise_images(iml, imr):
    """Testing.do_post, test.py:489-492: float32 z-normalisation."""
    imgl = iml.astype(np.float32)
    imgr = imr.astype(np.float32)
    imgl = (imgl - np.mean(imgl)) / np.std(imgl)
    imgr = (imgr - np.mean(imgr)) / np.std(imgr)
    return imgl, imgr


def postprocessing_mem(post, imgl, imgr, cost, direction, p=PARAMS):
    """Testing.__postprocessing_mem, test.py:341-449.  cost [H,W,D] f64."""
    post.InitCUDA()
    cross_array_init = np.zeros((4, imgl.shape[0], imgl.shape[1])).astype(np.float32)
    imgl_d = post.CUDA_float_array(imgl)
    imgr_d = post.CUDA_float_array(imgr)
    leftc_d = post.CUDA_float_array(cross_array_init)
    rightc_d = post.CUDA_float_array(cross_array_init)
    post.cross(imgl_d, leftc_d, p["L1"], p["tau1"])
    post.cross(imgr_d, rightc_d, p["L1"], p["tau1"])
    cost_d = post.CUDA_double_array(cost)
    temp_cost_d = post.CUDA_double_array(cost)
    post.swap_axis_back(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    for i in range(0, p["cbca_i1"]):
        post.cbca(leftc_d, rightc_d, cost_d, temp_cost_d, direction)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    post.swap_axis(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    tmp = np.zeros((cost.shape[1], cost.shape[2]))
    tmp_d = post.CUDA_double_array(tmp)
    for i in range(0, p["sgm_i"]):
        temp_cost_d.set_to_zero()
        tmp_d.set_to_zero()
        post.sgm(imgl_d, imgr_d, cost_d, temp_cost_d, tmp_d, p["pi1"], p["pi2"], p["tau_so"],
                 p["alpha1"], p["sgm_q1"], p["sgm_q2"], direction)
        post.CUDA_divide_double(temp_cost_d, 4)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    post.swap_axis_back(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    for i in range(0, p["cbca_i2"]):
        post.cbca(leftc_d, rightc_d, cost_d, temp_cost_d, direction)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    cc = cost_d.get_array()
    disp_l = np.argmin(cc, axis=0).astype(np.float32)
    disp_d = post.CUDA_float_array(disp_l)
    disp_temp = post.CUDA_float_array(disp_l)
    post.subpixel_enchancement(disp_d, cost_d, disp_temp)
    post.CUDA_copy_float(disp_temp, disp_d)
    for i in range(0, p["median_i"]):
        post.median2d(disp_d, disp_temp, p["median_w"])
        post.CUDA_copy_float(disp_temp, disp_d)
    post.mean2d(disp_d, disp_temp, gaussian(p["blur_sigma"]), p["blur_t"])
    post.CUDA_copy_float(disp_temp, disp_d)
    return disp_d.get_array()


def postprocessing_mem_interp(post, fte, imgl, imgr, cost, direction, p=PARAMS, check_outlier=None):
    """Testing.__postprocessing_mem_interp, test.py:153-338 (adds the
    right-reference chain and the left-right check).

    check_outlier(outlier) (optional) sees the outlier map before
    interpolate_mismatch runs; a backend with device-side asserts in that
    kernel (post.cu:810) needs every mismatch pixel to see a non-mismatch
    pixel along one of its 16 rays, and the caller checks that there."""
    r_cost = fte.get_right_cost(cost)
    post.InitCUDA()
    cross_array_init = np.zeros((4, imgl.shape[0], imgl.shape[1])).astype(np.float32)
    imgl_d = post.CUDA_float_array(imgl)
    imgr_d = post.CUDA_float_array(imgr)
    leftc_d = post.CUDA_float_array(cross_array_init)
    rightc_d = post.CUDA_float_array(cross_array_init)
    post.cross(imgl_d, leftc_d, p["L1"], p["tau1"])
    post.cross(imgr_d, rightc_d, p["L1"], p["tau1"])

    r_cost_d = post.CUDA_double_array(r_cost)
    temp_cost_d = post.CUDA_double_array(cost)
    tmp = np.zeros((cost.shape[1], cost.shape[2]))
    tmp_d = post.CUDA_double_array(tmp)
    post.swap_axis_back(r_cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, r_cost_d)
    for i in range(0, p["cbca_i1"]):
        post.cbca(rightc_d, leftc_d, r_cost_d, temp_cost_d, -1 * direction)
        post.CUDA_copy_double(temp_cost_d, r_cost_d)
    post.swap_axis(r_cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, r_cost_d)
    for i in range(0, p["sgm_i"]):
        temp_cost_d.set_to_zero()
        tmp_d.set_to_zero()
        post.sgm(imgl_d, imgr_d, r_cost_d, temp_cost_d, tmp_d, p["pi1"], p["pi2"], p["tau_so"],
                 p["alpha1"], p["sgm_q1"], p["sgm_q2"], -1 * direction)
        post.CUDA_divide_double(temp_cost_d, 4)
        post.CUDA_copy_double(temp_cost_d, r_cost_d)
    post.swap_axis_back(r_cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, r_cost_d)
    for i in range(0, p["cbca_i2"]):
        post.cbca(rightc_d, leftc_d, r_cost_d, temp_cost_d, -1 * direction)
        post.CUDA_copy_double(temp_cost_d, r_cost_d)
    cc = r_cost_d.get_array()
    r_disp = np.argmin(cc, axis=0).astype(np.float32)
    r_disp_d = post.CUDA_float_array(r_disp)

    cost_d = post.CUDA_double_array(cost)
    temp_cost_d = post.CUDA_double_array(cost)
    post.swap_axis_back(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    for i in range(0, p["cbca_i1"]):
        post.cbca(leftc_d, rightc_d, cost_d, temp_cost_d, direction)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    post.swap_axis(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    tmp = np.zeros((cost.shape[1], cost.shape[2]))
    tmp_d = post.CUDA_double_array(tmp)
    for i in range(0, p["sgm_i"]):
        temp_cost_d.set_to_zero()
        tmp_d.set_to_zero()
        post.sgm(imgl_d, imgr_d, cost_d, temp_cost_d, tmp_d, p["pi1"], p["pi2"], p["tau_so"],
                 p["alpha1"], p["sgm_q1"], p["sgm_q2"], direction)
        post.CUDA_divide_double(temp_cost_d, 4)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    post.swap_axis_back(cost_d, temp_cost_d)
    post.CUDA_copy_double(temp_cost_d, cost_d)
    for i in range(0, p["cbca_i2"]):
        post.cbca(leftc_d, rightc_d, cost_d, temp_cost_d, direction)
        post.CUDA_copy_double(temp_cost_d, cost_d)
    cc = cost_d.get_array()
    disp_l = np.argmin(cc, axis=0).astype(np.float32)
    out_s = cc.shape[0]
    disp_d = post.CUDA_float_array(disp_l)
    disp_temp = post.CUDA_float_array(disp_l)
    post.subpixel_enchancement(disp_d, cost_d, disp_temp)
    outlier = np.zeros((r_disp.shape[0], r_disp.shape[1])).astype(np.float32)
    outlier_d = post.CUDA_float_array(outlier)
    post.outlier_detection(disp_d, r_disp_d, outlier_d, out_s)
    if check_outlier is not None:
        check_outlier(outlier_d.get_array())
    post.interpolate_mismatch(disp_d, outlier_d, disp_temp)
    post.CUDA_copy_float(disp_temp, disp_d)
    post.interpolate_occlusion(disp_d, outlier_d, disp_temp)
    post.CUDA_copy_float(disp_temp, disp_d)
    post.CUDA_copy_float(disp_temp, disp_d)
    for i in range(0, p["median_i"]):
        post.median2d(disp_d, disp_temp, p["median_w"])
        post.CUDA_copy_float(disp_temp, disp_d)
    post.mean2d(disp_d, disp_temp, gaussian(p["blur_sigma"]), p["blur_t"])
    post.CUDA_copy_float(disp_temp, disp_d)
    return disp_d.get_array()


def eval_prob(post, fte, prob, iml, imr, d, interpolate=False, p=PARAMS, check_outlier=None):
    """Testing.eval_prob + do_post, test.py:143-149 and 485-504 (the
    graph-cut branch is out of scope).  Returns the disparity map."""
    h, w = iml.shape
    prob = np.reshape(prob, [h, w, d, 2])
    prob = fte.get_cost(prob)
    fte.get_right_cost(prob)  # computed by the reference, unused by _mem
    imgl, imgr = normalise_images(iml, imr)
    if interpolate:
        return postprocessing_mem_interp(post, fte, imgl, imgr, prob, -1, p, check_outlier)
    return postprocessing_mem(post, imgl, imgr, prob, -1, p)


def create_samples_mem(mtc, fte, iml, imr, gt, ndisp, d_indices):
    """Training.__create_samples_mem, train.py:100-273.

    gt: float disparity [H,W] (inf / negative = invalid).  d_indices(gt_int,
    ndisp) -> [S,3] int32 replaces fte.generate_d_indices (the reference's
    rand() inside OpenMP is not reproducible).  Returns samples [3S, 21]:
    20 features and the label."""
    h, w = iml.shape
    gt = np.reshape(gt, [gt.shape[0] * gt.shape[1], 1])
    infs = np.concatenate((np.argwhere(gt == np.inf), np.argwhere(gt < 0)), axis=0)
    gt = np.delete(gt, infs[:, 0], axis=0)
    gt = np.round(gt)
    gt = gt.astype(np.int32)
    random_samples = d_indices(gt, ndisp)
    samples = np.empty((random_samples.shape[0] * random_samples.shape[1], 21))
    cost = {}
    cost[0] = mtc.census(iml, imr, ndisp, 11).astype(np.float64)
    cost[1] = fte.swap_axes(mtc.nccNister(iml, imr, ndisp, 3))
    sobl = mtc.sobel(iml)
    sobr = mtc.sobel(imr)
    cost[2] = fte.swap_axes(mtc.sadsob(sobl, sobr, ndisp, 5).astype(np.float64))
    cost[3] = fte.swap_axes(mtc.zsad(iml, imr, ndisp, 5).astype(np.float64))
    es = (.01, 1.01, .01, .01)
    sig = (CENS_SIGMA, NCC_SIGMA, SAD_SIGMA, SAD_SIGMA)
    for k in range(4):
        c = cost[k]
        cR = fte.get_right_cost(c)
        c = np.reshape(c, [c.shape[0] * c.shape[1], c.shape[2]])
        cR = np.reshape(cR, [cR.shape[0] * cR.shape[1], cR.shape[2]])
        c = np.delete(c, infs[:, 0], axis=0)
        samples[:, k] = fte.get_samples(c, random_samples)
        samples[:, 4 + k] = fte.extract_ratio(c, random_samples, es[k])
        samples[:, 8 + k] = fte.extract_likelihood(c, random_samples, sig[k])
        r_pkrn = np.reshape(fte.extract_ratio(cR, es[k]), [h, w, ndisp])
        r_pkrn = fte.get_left_cost(r_pkrn)
        r_pkrn = np.reshape(r_pkrn, [r_pkrn.shape[0] * r_pkrn.shape[1], r_pkrn.shape[2]])
        r_pkrn = np.delete(r_pkrn, infs[:, 0], axis=0)
        samples[:, 12 + k] = fte.get_samples(r_pkrn, random_samples)
        r_aml = np.reshape(fte.extract_likelihood(cR, sig[k]), [h, w, ndisp])
        r_aml = fte.get_left_cost(r_aml)
        r_aml = np.reshape(r_aml, [r_aml.shape[0] * r_aml.shape[1], r_aml.shape[2]])
        r_aml = np.delete(r_aml, infs[:, 0], axis=0)
        samples[:, 16 + k] = fte.get_samples(r_aml, random_samples)
    samples[:, 20] = fte.generate_labels(random_samples)
    return samples
