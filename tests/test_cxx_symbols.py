"""The C++ overloads of tblis::mult over MArray DPD and indexed-DPD views are exported from
libtblis_b200_cxx.so under the mangled names TBLIS's own library exports
(src/iface/3t/mult.cxx:292-298 instantiates float, double, scomplex and
dcomplex), so a C++ program built against TBLIS links to them unchanged."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX_LIB = os.path.join(ROOT, "tblis_b200", "libtblis_b200_cxx.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtblis_ref.so")

# tblis::mult<T>(tci::communicator const&, T, MArray::dpd_varray_view<T const>,
# char const*, MArray::dpd_varray_view<T const>, char const*, T,
# MArray::dpd_varray_view<T>, char const*)
DPD_MULT = [
    "_ZN5tblis4multIfEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIKS5_EEPKcS9_SB_S5_NS7_IS5_EESB_",
    "_ZN5tblis4multIdEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIKS5_EEPKcS9_SB_S5_NS7_IS5_EESB_",
    "_ZN5tblis4multISt7complexIfEEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIKS7_EEPKcSB_SD_S7_NS9_IS7_EESD_",
    "_ZN5tblis4multISt7complexIdEEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIKS7_EEPKcSB_SD_S7_NS9_IS7_EESD_",
]


# the same for MArray::indexed_dpd_varray_view (src/iface/3t/mult.cxx:535-541)
INDEXED_DPD_MULT = [n.replace("15dpd_varray_view", "23indexed_dpd_varray_view") for n in DPD_MULT]


# the DPD level-1 overloads (src/iface/1t/{add,dot,reduce,scale,set,shift}.cxx), double
DPD_LEVEL1 = [
    "_ZN5tblis3addIdEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIKS5_EEPKcS5_NS7_IS5_EESB_",
    "_ZN5tblis3dotIdEEvRKN3tci12communicatorEN6MArray15dpd_varray_viewIKT_EEPKcS9_SB_RS7_",
    "_ZN5tblis6reduceIdEEvRKN3tci12communicatorENS_8reduce_tEN6MArray15dpd_varray_viewIKT_EEPKcRS8_Rl",
    "_ZN5tblis5scaleIdEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIS5_EEPKc",
    "_ZN5tblis3setIdEEvRKN3tci12communicatorET_N6MArray15dpd_varray_viewIS5_EEPKc",
    "_ZN5tblis5shiftIdEEvRKN3tci12communicatorET_S5_N6MArray15dpd_varray_viewIS5_EEPKc",
]


INDEXED_DPD_LEVEL1 = [n.replace("15dpd_varray_view", "23indexed_dpd_varray_view") for n in DPD_LEVEL1]


def _has(lib, name):
    try:
        getattr(lib, name)
        return True
    except AttributeError:
        return False


def test_cxx_library_exports_the_dpd_overloads():
    assert os.path.exists(CXX_LIB), "libtblis_b200_cxx.so not built (make -C tblis_b200 cxx MARRAY=...)"
    lib = ctypes.CDLL(CXX_LIB, mode=ctypes.RTLD_LOCAL)
    missing = [n for n in DPD_MULT + INDEXED_DPD_MULT + DPD_LEVEL1 + INDEXED_DPD_LEVEL1 if not _has(lib, n)]
    assert not missing, missing


def test_names_match_the_reference_library():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built here")
    ref = ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_LOCAL)
    assert all(_has(ref, n) for n in DPD_MULT + INDEXED_DPD_MULT + DPD_LEVEL1 + INDEXED_DPD_LEVEL1)
