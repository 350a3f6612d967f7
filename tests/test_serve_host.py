"""The request server's scheduler (tsunami_pact_b200/csrc/tsu_serve.h) on the
CPU, over a fake executor (tests/serve/sched_driver.cpp), built with
ThreadSanitizer: admission against the memory budget, FIFO start order,
merging of queued requests into jobs, long pairs as jobs of their own,
result splitting and reassembly, cancellation,
pending/overflow polls, the watchdog, retries after memory failures, failure
isolation, the queue limit, many client threads at once and shutdown.
Failures are made on the host (a fake that sleeps, fails or asks for more
memory); nothing here touches a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "serve", "sched_driver.cpp")
HDRS = [os.path.join(ROOT, "tsunami_pact_b200", "csrc", f) for f in ("tsu_serve.h", "tsu_estimate.h")] + [
    os.path.join(ROOT, "include", "tsunami_b200.h")]
EXE = os.path.join(ROOT, "tests", "serve", "_build", "sched_driver")

SCENARIOS = ["basic", "score_only", "admission", "concurrency", "reject", "degraded", "fifo", "cancel", "pending",
             "watchdog", "nomem_retry", "failure_isolation", "queue_full", "stress", "shutdown", "heavy_split",
             "heavy_fail", "estimate", "lowmem"]


@pytest.fixture(scope="module")
def driver():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    newest = max(os.path.getmtime(s) for s in [SRC] + HDRS)
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < newest:
        # built under a per-process name and renamed into place, so parallel
        # pytest workers never run a half-written binary
        tmp_exe = f"{EXE}.tmp{os.getpid()}"
        subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=thread", "-o", tmp_exe, SRC, "-lpthread"],
                       check=True)
        os.replace(tmp_exe, EXE)
    return EXE


@pytest.mark.parametrize("scenario", SCENARIOS)
def test_scheduler(driver, scenario):
    env = dict(os.environ, TSAN_OPTIONS="halt_on_error=1 second_deadlock_stack=1")
    r = subprocess.run([driver, scenario], capture_output=True, timeout=120, env=env)
    assert r.returncode == 0, (r.stdout.decode() + r.stderr.decode())[-4000:]
    assert r.stdout.decode().strip() == f"ok {scenario}"
