"""The generated FFT plan table and instantiation files are what the
generator produces (CPU): regenerating them in a scratch copy changes
nothing, so the committed kernels and their launch shapes stay in step."""
import filecmp
import os
import shutil
import subprocess
import sys

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "deconwolf_b200", "csrc")


def test_generated_files_are_current(tmp_path):
    shutil.copy(os.path.join(CSRC, "gen_plans.py"), tmp_path)
    subprocess.run([sys.executable, "gen_plans.py", "--parts", "16"], cwd=tmp_path, check=True,
                   capture_output=True)
    made = sorted(f for f in os.listdir(tmp_path) if f.startswith("inst_") or f == "plans_gen.h")
    have = sorted(f for f in os.listdir(CSRC) if (f.startswith("inst_") and f.endswith(".cu")) or f == "plans_gen.h")
    assert made == have
    for f in made:
        assert filecmp.cmp(os.path.join(tmp_path, f), os.path.join(CSRC, f), shallow=False), f
    # the y pass's translation units keep scalar complex adds
    for f in made:
        if f.startswith("inst_y_"):
            assert "#define DW_PAIRED_ADDS 0" in open(os.path.join(CSRC, f)).read()
