"""Extracts the modified Shepp-Logan ellipsoid table (10 rows x A, a, b, c, x0, y0, z0,
phi, theta, psi) from TomoGPI's Data3D_0256/phantom3d.m (function modified_shepp_logan)
and writes it to modified_shepp_logan.txt beside this script. Run where the TomoGPI source
tree is available:  python tomogpi_b200/data/make_shepp_logan_table.py <TomoGPI>/Data3D_0256/phantom3d.m
"""
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: make_shepp_logan_table.py <path to TomoGPI's Data3D_0256/phantom3d.m>")
src = Path(sys.argv[1])
text = src.read_text()
body = text.split("function e = modified_shepp_logan", 1)[1].split("return;", 1)[0]
block = body.split("e =", 1)[1].split("];", 1)[0].replace("[", " ")
rows = []
for line in block.strip().splitlines():
    nums = re.findall(r"[-+]?(?:\d+\.?\d*|\.\d+)", line)
    if len(nums) == 10:
        rows.append(nums)
assert len(rows) == 10, rows
out = Path(__file__).resolve().parent / "modified_shepp_logan.txt"
with out.open("w") as fh:
    fh.write("# modified Shepp-Logan (phantom3d.m, modified_shepp_logan): A a b c x0 y0 z0 phi theta psi\n")
    for r in rows:
        fh.write(" ".join(r) + "\n")
print(out)
