"""KDE oracle restatement against the reference's own kde.cl kernels (CPU only)."""
import numpy as np
import pytest

import oracle as O
from kde_cases import bivariate, univariate

needs_ref = pytest.mark.skipif(not O.ref_available("histogram_univariate"),
                               reason="reference kernels not compiled (oracle/_ref)")
SHAPES = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]


@needs_ref
@pytest.mark.parametrize("kind", SHAPES)
@pytest.mark.parametrize("nb,npp", [(2048, 256), (8192, 1024), (1000, 100)])
def test_univariate_vs_reference(kind, nb, npp):
    d, prm = univariate(kind, n_hist_bins=nb, n_pdf_points=npp)
    data = np.ascontiguousarray(d.logx_data.reshape(-1), dtype=np.float32)
    h = O.histogram_univariate(prm, data)
    rh = O.ref_kde("histogram_univariate", prm, data, nb, np.uint32, data.size)
    assert np.array_equal(h, rh)
    assert int(h.sum()) == data.size
    pdf = O.pdf_univariate(prm, h)
    rpdf = O.ref_kde("pdf_univariate", prm, h, npp, np.float32, npp)
    assert np.array_equal(pdf.view(np.uint32), rpdf.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("kind", SHAPES)
def test_bivariate_vs_reference(kind):
    d, prm = bivariate(kind)
    nb, npp = int(d.n_hist_bins), int(d.n_pdf_points)
    data = np.ascontiguousarray(d.logxy_data, dtype=np.float32)
    h = O.histogram_bivariate(prm, data)
    rh = O.ref_kde("histogram_bivariate", prm, data, nb * nb, np.uint32, data.shape[0])
    assert np.array_equal(h, rh)
    part = O.pdf_bivariate_rows(prm, h)
    rpart = O.ref_kde("pdf_bivariate_rows", prm, h, nb * nb, np.float32, nb * nb)
    assert np.array_equal(part.view(np.uint32), rpart.view(np.uint32))
    pdf = O.pdf_bivariate_cols(prm, part)
    rpdf = O.ref_kde("pdf_bivariate_cols", prm, part, npp * npp, np.float32, npp * npp)
    assert np.array_equal(pdf.view(np.uint32), rpdf.view(np.uint32))
    assert np.isfinite(pdf).all() and pdf.max() > 0
