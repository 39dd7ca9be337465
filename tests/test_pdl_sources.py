"""Every kernel launched with programmatic dependent launch (BN_LAUNCH_PDL)
begins with BN_PDL_ENTRY(), the wait for the previous kernel's results:
without it the kernel could read data that the kernel before it has not
written yet."""
import glob
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "blood_network_b200", "csrc")


def _kernel_body_start(src, name):
    m = re.search(r"__global__[^;{]*?\b" + re.escape(name) + r"\s*\(", src)
    if not m:
        return None
    i, depth = m.end() - 1, 0
    while True:
        if src[i] == "(":
            depth += 1
        elif src[i] == ")":
            depth -= 1
            if depth == 0:
                break
        i += 1
    j = src.index("{", i)
    return src[j + 1:j + 200]


def test_pdl_launched_kernels_wait_first():
    sources = {f: open(f).read() for f in glob.glob(os.path.join(CSRC, "*.cu"))}
    every = "".join(sources.values())
    launched = set()
    for src in sources.values():
        for m in re.finditer(r"BN_LAUNCH_PDL\(\(?\s*([A-Za-z_][A-Za-z0-9_]*)", src):
            launched.add(m.group(1))
    assert len(launched) >= 20
    for name in sorted(launched):
        body = _kernel_body_start(every, name)
        assert body is not None, name
        assert body.lstrip().startswith("BN_PDL_ENTRY();"), name
