"""The product's planar geometry (the mesh's Delaunay triangulation, triangle
affine maps, point-in-triangle distances, hull area, the homography refit)
against the oracle's own code for the same rules, on seeded point sets that
include full lattices (every cell co-circular) and anchor lattices with holes:
the same triangles in the same vertex order, and the same bits from every
floating-point helper. CPU only."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_product_geometry_matches_oracle(tmp_path):
    exe = str(tmp_path / "geom_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    "-I", os.path.join(REPO, "semper-dic-engine_b200", "csrc", "host"),
                    "-I", os.path.join(REPO, "oracle", "src"),
                    os.path.join(REPO, "tests", "cpp", "geom_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-2000:]
    assert r.stdout.strip().endswith("same")
