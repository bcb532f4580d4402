"""The native build's steps rerun when their inputs' contents or command change, and only then; a copy of the
tree elsewhere reuses its built files (no GPU, no compiler: the steps here are small Python commands)."""
import os
import shutil
import sys

from galn_b200 import build


def _write(p, s):
    with open(p, "w") as f:
        f.write(s)


def _step(tmp, name="out.txt", flag="a"):
    src, out = os.path.join(tmp, "in.txt"), os.path.join(tmp, name)
    cmd = [sys.executable, "-c", f"import shutil; shutil.copy({src!r}, {out!r})", flag]
    ran = []
    real = build.subprocess.run

    def counting(c, check):
        ran.append(c)
        return real(c, check=check)

    build.subprocess.run = counting
    try:
        build._step(out, cmd, [src], False)
    finally:
        build.subprocess.run = real
    return len(ran), out


def test_step_reruns_on_content_and_flags_only(tmp_path, monkeypatch):
    monkeypatch.setattr(build, "ROOT", str(tmp_path))
    _write(tmp_path / "in.txt", "one")
    assert _step(str(tmp_path))[0] == 1
    assert _step(str(tmp_path))[0] == 0                      # nothing changed
    os.utime(tmp_path / "in.txt", (1, 1))                   # an older time, same contents: still nothing
    assert _step(str(tmp_path))[0] == 0
    _write(tmp_path / "in.txt", "two")
    n, out = _step(str(tmp_path))
    assert n == 1 and open(out).read() == "two"
    assert _step(str(tmp_path), flag="b")[0] == 1            # a changed command line
    os.remove(out)
    assert _step(str(tmp_path), flag="b")[0] == 1            # a missing output


def test_copied_tree_reuses_its_outputs(tmp_path, monkeypatch):
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    _write(a / "in.txt", "x")
    monkeypatch.setattr(build, "ROOT", str(a))
    assert _step(str(a))[0] == 1
    shutil.copytree(a, b)
    monkeypatch.setattr(build, "ROOT", str(b))
    assert _step(str(b))[0] == 0
