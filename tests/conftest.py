import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "wukong-cube_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "refpin"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built():
    """Build the product library and the oracle once per session."""
    import wk_build as wkbuild
    wkbuild.build_lib()
    wkbuild.build_synth()
    wkbuild.build_oracle()
    return True


@pytest.fixture(scope="session")
def graph20(built):
    """The 20-organisation synthetic graph, its host store and the oracle store."""
    import oracle
    import wukong_b200 as wk
    tr, v = wk.synth_generate(20, seed=0)
    g = wk.GStore(tr)
    o = oracle.OracleStore(tr)
    inst = {t: g.get_index(t, wk.IN) for t in range(v["t_org"], v["t_doc"] + 1)}
    return {"triples": tr, "vocab": v, "gstore": g, "oracle": o, "instances": inst}


@pytest.fixture(scope="session")
def ctx(graph20):
    import wukong_b200 as wk
    c = wk.Context(0)
    c.upload_gstore(graph20["gstore"])
    yield c
    c.close()
