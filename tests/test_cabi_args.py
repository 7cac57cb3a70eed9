"""Host-side faults through the C ABI, without a GPU: null pointers and sizes
out of range come back as ORBX_ERR_ARG / ORBX_ERR_SIZE before any CUDA call,
and nothing exits the process.  Device pointers passed here are never
dereferenced: each call is rejected by its argument checks first."""
import ctypes

import pytest

import orbx

FAKE = ctypes.c_void_p(16)  # a non-null stand-in, never dereferenced


@pytest.fixture(scope="module")
def L():
    return orbx.lib()


def test_status_strings_distinct(L):
    names = [orbx.status_string(s) for s in range(7)]
    assert all(names) and len(set(names)) == 7


def test_knn2_argument_checks(L):
    assert L.orbx_match_knn2(None, FAKE, 1, FAKE, 1, FAKE, FAKE, 0) == orbx.ORBX_ERR_ARG
    assert L.orbx_match_knn2_static(FAKE, -1, FAKE, 1, FAKE, FAKE, None) == orbx.ORBX_ERR_ARG
    assert L.orbx_match_knn2_static(None, 4, FAKE, 1, FAKE, FAKE, None) == orbx.ORBX_ERR_ARG
    assert L.orbx_match_knn2_static(FAKE, 4, None, 1, FAKE, FAKE, None) == orbx.ORBX_ERR_ARG
    assert (L.orbx_match_knn2_static(FAKE, 16385, FAKE, 1, FAKE, FAKE, None) == orbx.ORBX_ERR_SIZE)
    assert (L.orbx_match_knn2_static(FAKE, 1, FAKE, 1 << 22, FAKE, FAKE, None) == orbx.ORBX_ERR_SIZE)
    assert L.orbx_match_knn2_static(None, 0, None, 0, None, None, None) == orbx.ORBX_OK  # nothing to do


def test_learned_argument_checks(L):
    p = orbx.LearnedParams()
    assert L.orbx_learned_default_params(None) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_default_params(ctypes.byref(p)) == orbx.ORBX_OK
    assert (p.proposal, p.n_clusters, p.hidden, p.n_probe) == (orbx.PROPOSAL_MLP, 4096, 512, 8)
    assert (p.rerank, p.label_mode) == (orbx.RERANK_TENSOR, orbx.LABEL_LISTED)
    h = ctypes.c_void_p()
    assert L.orbx_learned_build(None, ctypes.byref(p), FAKE, 100, FAKE, 100, ctypes.byref(h)) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_set_margin(None, ctypes.c_float(0.0)) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_set_max_distance(None, 10) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_set_rerank(None, orbx.RERANK_POPC) == orbx.ORBX_ERR_ARG
    need = ctypes.c_size_t()
    assert L.orbx_learned_save(None, None, None, 0, ctypes.byref(need)) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_load(None, FAKE, 100, FAKE, 10, ctypes.byref(h)) == orbx.ORBX_ERR_ARG
    assert L.orbx_learned_destroy(None) == orbx.ORBX_ERR_ARG
    st = orbx.LearnedStats()
    assert L.orbx_learned_get_stats(None, ctypes.byref(st)) == orbx.ORBX_ERR_ARG


def test_gemm_and_ocv_argument_checks(L):
    assert L.orbx_gemm_bf16(None, FAKE, FAKE, 128, 256, 64, None, 0, 1, FAKE, None) == orbx.ORBX_ERR_ARG
    assert L.orbx_ocv_default_params(None) == orbx.ORBX_ERR_ARG
