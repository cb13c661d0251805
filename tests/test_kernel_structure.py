"""Static check of the column kernel's warp-level control skeleton (no GPU needed).

The FP64 column code (uw_column, which every kernel runs) joins the live lanes of a warp with
__syncwarp(live) (the UW_SYNC() macro).  That is only well defined if every live lane executes the
same sequence of UW_SYNC() calls, so each call
must sit directly inside blocks that all live lanes enter equally often: the function body, the
`if (active)` block, plain `{ }` blocks, and loops marked `// uniform` (same trip count on every
lane).  Such a loop must also have no `break` or `continue` of its own, which would let some lanes
leave it or skip its UW_SYNC().  This test parses the kernel's braces and checks both rules."""
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KERNEL = os.path.join(REPO, "hpc-and-climate-model_b200", "csrc", "uwshcu_fp64_kernel.cuh")


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), text, flags=re.S)
    return text


def _scan():
    raw = open(KERNEL).read().split("\n")
    code = _strip_comments("\n".join(raw)).split("\n")
    stack = []            # (line number, opener text, kind) for each open brace
    syncs, jumps = [], []
    in_kernel = False
    for ln, (line, rline) in enumerate(zip(code, raw), 1):
        body = line.split("//")[0]
        if "void uw_column(" in body:
            in_kernel = True
        if not in_kernel:
            continue
        uniform = rline.rstrip().endswith("// uniform")
        pos = 0
        for m in re.finditer(r"[{}]|UW_SYNC\(\);|\bbreak;|\bcontinue;", body):
            tok = m.group(0)
            prefix = body[pos:m.start()]
            if tok == "{":
                head = body[: m.start()].strip()
                if re.search(r"\bdo$", head):
                    kind = "loop"
                elif re.match(r"(\}\s*)?(for|while)\s*\(", head):
                    kind = "loop"
                elif head == "" or head.endswith(";"):
                    kind = "block"
                else:
                    kind = "branch"
                stack.append((ln, head, kind, uniform))
            elif tok == "}":
                if stack:
                    stack.pop()
                if in_kernel and not stack:
                    return syncs, jumps
            elif tok == "UW_SYNC();":
                syncs.append((ln, list(stack)))
            else:
                # innermost loop this statement belongs to; a braceless `if (...) break;` counts
                # as inside that loop too
                jumps.append((ln, tok, list(stack)))
            pos = m.end()
    return syncs, jumps


def _allowed(entry):
    ln, head, kind, uniform = entry
    if "uw_column(" in head:
        return True
    if head == "if (active)":
        return True
    if kind == "block":
        return True
    return uniform


def test_every_warp_sync_is_reached_uniformly():
    syncs, _ = _scan()
    assert len(syncs) >= 10
    bad = []
    for ln, stack in syncs:
        # the kernel function's own brace is the first entry
        for entry in stack[1:]:
            if not _allowed(entry):
                bad.append((ln, entry[0], entry[1]))
    assert not bad, "UW_SYNC() under a lane-dependent block: %s" % bad


def test_uniform_loops_have_no_lane_dependent_exit():
    _, jumps = _scan()
    bad = []
    for ln, tok, stack in jumps:
        loops = [e for e in stack if e[2] == "loop"]
        if loops and loops[-1][3]:
            bad.append((ln, tok, loops[-1][0]))
    assert not bad, "break/continue inside a uniform loop: %s" % bad


def test_uniform_loops_are_marked():
    syncs, _ = _scan()
    marked = set()
    for _, stack in syncs:
        for e in stack:
            if e[3]:
                marked.add(e[1].split("(")[0].strip())
    assert {"for"} <= marked or {"for", "if"} <= marked, marked
