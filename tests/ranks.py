"""Start the ranks of a multi-process test: one `python -m tests.ranks_worker`
process per rank with MINIMPI_SIZE / MINIMPI_RANK / MINIMPI_DIR set (the
stand-in MPI library joins them over Unix sockets in that directory), wait
for all with a bound, and report each rank's exit status and output."""
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_ranks(size, scenario, device=False, timeout=180, env_extra=None):
    """(returncodes, outputs) of `size` ranks running `scenario`; ranks still
    running at `timeout` seconds are killed (their exact PIDs)."""
    with tempfile.TemporaryDirectory(prefix="minimpi-") as d:
        procs = []
        for r in range(size):
            env = dict(os.environ, MINIMPI_SIZE=str(size), MINIMPI_RANK=str(r), MINIMPI_DIR=d,
                       MINIMPI_TIMEOUT_S="60", PYTHONPATH=ROOT)
            env.update(env_extra or {})
            args = [sys.executable, "-m", "tests.ranks_worker", scenario]
            if device:
                args.append("device")
            procs.append(subprocess.Popen(args, cwd=ROOT, env=env, stdout=subprocess.PIPE,
                                          stderr=subprocess.STDOUT, text=True))
        t0 = time.time()
        outs = [None] * size
        for i, p in enumerate(procs):
            try:
                outs[i], _ = p.communicate(timeout=max(1.0, timeout - (time.time() - t0)))
            except subprocess.TimeoutExpired:
                for q in procs:
                    if q.poll() is None:
                        q.kill()
                outs[i], _ = p.communicate()
        return [p.returncode for p in procs], outs
