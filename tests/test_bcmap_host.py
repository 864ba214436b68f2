"""The boundary-copy map of the whole-step kernels (mage_b200/csrc/gam_bcmap.cuh),
compiled for the host with g++ (no GPU):

* its composed source index equals the PyTorch restatement's
  (mage_b200.diffstep.Grid._bc_maps) at every box position, for cells and the
  three face directions, periodic and zero-gradient J, with periodic I and
  with the non-periodic I sides (whose fills run before the gather);
* the tables of the gather's adjoint (bc_adj_tables) list for each position
  exactly the positions the map copies from it, in ascending order
  (brute-force preimages), and flag the positions the map fixes.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mage_b200.diffstep import DiffParams, Grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cstdio>
#include <cstdlib>
#include "gam_bcmap.cuh"
using namespace gam_stepadj;
int main(int argc, char** argv) {
    gam_params p{};
    p.Nip = atoi(argv[1]); p.Njp = atoi(argv[2]); p.Nkp = atoi(argv[3]);
    for (int q = 0; q < 6; q++) p.bc[q] = atoi(argv[4 + q]);
    const Box b = make_box(&p);
    for (int comp = -1; comp < 3; comp++)
        for (int k = 0; k < b.nz; k++) for (int j = 0; j < b.ny; j++) for (int i = 0; i < b.nx; i++)
            printf("%ld\n", bc_source(b, comp, i, j, k));
    for (int comp = -1; comp < 3; comp++) {
        std::vector<int> code, rowStart, src;
        bc_adj_tables(b, comp, code, rowStart, src);
        for (long s = 0; s < b.n; s++) {
            const int row = (code[s] >> 1) - 1;
            printf("P %d %ld %d", comp, s, code[s] & 1);
            if (row >= 0)
                for (int q = rowStart[row]; q < rowStart[row + 1]; q++) printf(" %d", src[q]);
            printf("\n");
        }
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not available")
    d = tmp_path_factory.mktemp("bcmap")
    src = d / "bcmap.cpp"
    src.write_text(HARNESS)
    exe = d / "bcmap"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "mage_b200", "csrc"), "-o", str(exe),
                    str(src)], check=True)
    return str(exe)


class _Box:
    """The attributes Grid._bc_maps reads, without geometry."""

    def __init__(self, N, bc):
        self.P = DiffParams(*N, bc=bc)
        self.Ni, self.Nj, self.Nk = N[0] + 8, N[1] + 8, N[2] + 8
        self.device = "cpu"


@pytest.mark.parametrize("N", [(16, 16, 16), (16, 24, 8), (8, 4, 4), (4, 6, 5)])
@pytest.mark.parametrize("bc", [(0, 0, 0, 0, 0, 0), (0, 0, 2, 2, 0, 0), (3, 4, 2, 2, 0, 0), (6, 2, 0, 0, 0, 0)],
                         ids=["periodic", "zerogradJ", "sphin-wind-zerogradJ", "inflow-obcI"])
def test_bc_map_matches_restatement(harness, N, bc):
    out = subprocess.run([harness, *map(str, N), *map(str, bc)], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    n = (N[0] + 9) * (N[1] + 9) * (N[2] + 9)
    src = np.array([int(x) for x in out[:4 * n]]).reshape(4, n)
    box = _Box(N, bc)
    Grid._bc_maps(box)
    for c, comp in enumerate((-1, 0, 1, 2)):
        assert np.array_equal(src[c], box.bc_src[comp].numpy()), comp
    idx = np.arange(n)
    for line in out[4 * n:]:
        if not line.startswith("P"):
            continue
        f = line.split()
        c, s, fixed = int(f[1]), int(f[2]), int(f[3])
        got = [int(x) for x in f[4:]]
        m = src[c + 1]
        want = idx[(m == s) & (idx != s)].tolist()
        assert got == want, (c, s, got, want)
        assert fixed == int(m[s] == s), (c, s)
