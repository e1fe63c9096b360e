import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def load_fixture(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def fixture_names() -> list[str]:
    return sorted(p.name for p in GOLDEN.glob("*.json"))


def host_graph_from_fixture(fx: dict):
    from gpugraph_b200 import HostGraph

    if "row_offsets" in fx:
        return HostGraph(np.asarray(fx["row_offsets"], np.int32), np.asarray(fx["column_indices"], np.int32),
                         np.asarray(fx["edge_values"], np.int32), directed=True)
    g = HostGraph.rmat(fx["scale"], fx["edgefactor"], seed=fx["seed"], symmetrize=fx["symmetrize"])
    return g.with_weights(1, 64, seed=fx["seed"])


@pytest.fixture(scope="session")
def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
