"""Every kernel started through vtp::launch waits for its predecessor first.

vtp::launch (csrc/common.cuh) may add the programmatic-stream-serialization
attribute, which lets a kernel's blocks start while the kernel before it in
the stream is still running.  Stream order then holds only because each such
kernel's first statement is pdl_enter() (griddepcontrol.wait).  A kernel
routed through launch() without it would race with its predecessor; this
CPU test reads the CUDA sources and fails on any such kernel.
"""
import re
from pathlib import Path

CSRC = Path(__file__).resolve().parent.parent / "vt-physics_b200" / "csrc"

_LAUNCH = re.compile(r"\blaunch\(\s*(?:vtp::)?([A-Za-z_]\w*)")


def _kernel_bodies(text):
    """Map kernel name -> source text of its body, for every __global__ definition."""
    out = {}
    for m in re.finditer(r"__global__\s+void\s+(?:__launch_bounds__\([^)]*\)\s*)?([A-Za-z_]\w*)\s*\(", text):
        name = m.group(1)
        # Skip the parameter list, then take the body if this is a definition.
        i = m.end()
        depth = 1
        while depth:
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        rest = text[i:].lstrip()
        if not rest.startswith("{"):
            continue   # a declaration
        out.setdefault(name, rest[1:400])
    return out


def test_every_launch_helper_kernel_starts_with_pdl_enter():
    texts = {p.name: p.read_text() for p in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh"))}
    bodies = {}
    for t in texts.values():
        for k, v in _kernel_bodies(t).items():
            bodies.setdefault(k, v)
    launched = set()
    for name, t in texts.items():
        for m in _LAUNCH.finditer(t):
            if name == "common.cuh":
                continue   # the helper's own definition
            launched.add(m.group(1))
    assert len(launched) >= 15, sorted(launched)
    missing = []
    for k in sorted(launched):
        assert k in bodies, f"kernel {k} passed to launch() has no __global__ definition in csrc/"
        first = bodies[k].split(";")[0].strip()
        if first != "pdl_enter()" and first != "vtp::pdl_enter()":
            missing.append((k, first))
    assert not missing, f"kernels launched through launch() without pdl_enter() first: {missing}"
