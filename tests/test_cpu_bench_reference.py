"""The reference arm of bench.py runs the oracle's PIC steps on the host cores
alone: it prints one JSON line with the contract's keys and the same config
object as the GPU arm, never loads the CUDA library, and under torchrun only
rank 0 prints. Run on the small workload A so that it takes seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1", "--workload", "A"]

# runs bench.py in this interpreter, then reports whether any in-tree CUDA
# library was mapped into the process
PROBE = """
import runpy, sys
sys.argv = %r
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
maps = open("/proc/self/maps").read()
print("LIBWARP_MAPPED=%%d" %% ("libwarp_b200.so" in maps))
print("LIB_MODULE=%%d" %% ("warp_b200._lib" in sys.modules))
""" % (ARGS,)


def _run(env):
    return subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=600, check=True)


def test_reference_arm_prints_the_contract_line_without_the_library():
    env = dict(os.environ, ORACLE_THREADS="2")
    env.pop("RANK", None)
    out = _run(env)
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert lines[-2:] == ["LIBWARP_MAPPED=0", "LIB_MODULE=0"]
    assert len(lines) == 3
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] == 2
    # the timed steps are real: ms_per_step covers whole oracle steps with
    # their own V-cycle counts
    assert d["vcycles_per_solve"] >= 1
    assert d["ms_per_step"] * d["steps"] < 600e3
    # the same config object as the GPU arm prints for this workload
    sys.path.insert(0, ROOT)
    import bench
    from warp_b200.workloads import workload
    assert d["config"] == bench.job_config(workload("A"), 1)
    assert d["config"]["workload"].startswith("32x32x64")


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = _run(env)
    assert [ln for ln in out.stdout.splitlines() if ln.strip()] == ["LIBWARP_MAPPED=0", "LIB_MODULE=0"]
