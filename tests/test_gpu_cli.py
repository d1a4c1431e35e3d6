"""The CLI as a drop-in for test_lu.pl (test_lu.pl:9-84): every parameter
set of its five tables (block sizes, pivot agglomeration batch sizes,
mapping arguments, medium and large sizes) through
`python -m charmlu_b200 N b mem [batch mapping ...]`, graded the way
test_lu.pl grades it: the `residual = X` line must give X < 16."""
import os
import re
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# test_lu.pl's tables: smalltests, agglomtests, mappingtests, mediumtests, largetests
TEST_LU_PL_ARGS = [
    [48, 48, 500], [48, 24, 500], [48, 16, 500], [48, 12, 500],
    [32, 8, 500, 9], [32, 8, 500, 8], [32, 8, 500, 7], [32, 8, 500, 4], [32, 8, 500, 3], [32, 8, 500, 2],
    [32, 8, 500, 1], [32, 4, 500, 2], [32, 4, 500, 1],
    [512, 128, 500, 128, 2], [512, 128, 500, 128, 3], [512, 64, 500, 128, 3, 4, 1],
    [512, 64, 500, 128, 3, 4, 1, 1], [512, 64, 500, 128, 3, 4, 1, 2], [512, 64, 500, 128, 3, 1, 4, 2, 4],
    [512, 64, 500, 128, 3, 1, 4, 2, 2], [512, 64, 500, 128, 3, 1, 4, 2, 1],
    [512, 256, 500], [512, 128, 500], [1024, 256, 500], [1024, 128, 500], [1024, 64, 500],
    [2048, 256, 500], [2048, 512, 500], [4096, 256, 500], [4096, 512, 500],
]
RESIDUAL = re.compile(r"residual = ([\d\.]*)")  # test_lu.pl:77


# every line the reference prints around a solve (benchmark.C:150-184, 343-400)
FLOAT = r"[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|inf|nan)"
REF_LINES = [
    r"^Running LU compiled from revision: \S+$",
    r"^Running LU on \d+ processors \(\d+ nodes\): $",
    r"^\tMatrix size: \d+ X \d+ $",
    r"^\tBlock size: \d+ X \d+ $",
    r"^\tChare Array size: \d+ X \d+$",
    r"^\tPivot batch size: \d+$",
    r"^\tMem Threshold \(MB\): \d+$",
    r"^\tSend Limit: \d+$",
    r"^\tMapping Scheme: \d+ \((Block Cyclic|2D Tiling)\)$",
    r"^\tPivot Redn Scheduling: (On|Off)$",
    r"^\tUseg Multicast from: (Below|Diagonal)$",
    r"^RESULT procs: \t\d+\tblock size:\t\d+\tTime\(s\):\t" + FLOAT + "$",
    r"^HPL flop count gives \t" + FLOAT + r"\tGFlops$",
    r"^Order:\t" + FLOAT + "% of peak$",
    r"^Abe:\t" + FLOAT + "% of peak$",
    r"^Ranger:\t" + FLOAT + "% of peak$",
    r"^Jaguar/Kraken XT5:\t" + FLOAT + "% of peak$",
    r"^BG/P:\t" + FLOAT + "% of peak$",
    r"^Jaguar XK6 sans GPUs:\t" + FLOAT + "% of peak$",
    r"^The dgemm \d+ x \d+ takes " + FLOAT + " ms and achieves " + FLOAT + " GFlop/sec$",
    r"^Percent of DGEMM is: " + FLOAT + "%$",
    r"^epsilon = \d\.\d{6}e[-+]\d+$",
    r"^residual = \d+\.\d{6}$",
    r"^finished validation at wall time: \d+\.\d{6}$",
]


@pytest.mark.parametrize("args", TEST_LU_PL_ARGS, ids=lambda a: "_".join(map(str, a)))
def test_cli_residual_line(cuda_dev, capsys, args):
    from charmlu_b200.__main__ import main
    assert main([str(v) for v in args]) in (0, None)
    out = capsys.readouterr().out
    m = RESIDUAL.search(out)
    assert m is not None, out
    assert float(m.group(1)) < 16, out
    assert "RESULT procs:" in out and "HPL flop count gives" in out
    assert f"Pivot batch size: {args[3] if len(args) > 3 else args[1] // 4}" in out


@pytest.mark.parametrize("args", [[512, 128, 500], [512, 64, 500, 128, 3, 4, 1, 2]],
                         ids=lambda a: "_".join(map(str, a)))
def test_cli_prints_every_reference_line(cuda_dev, capsys, args):
    """Each result and configuration line of the reference has its
    counterpart, in the reference's format, in the reference's order."""
    from charmlu_b200.__main__ import main
    assert main([str(v) for v in args]) in (0, None)
    lines = capsys.readouterr().out.splitlines()
    pos = -1
    for pat in REF_LINES:
        hits = [i for i, ln in enumerate(lines) if re.match(pat, ln)]
        assert hits, (pat, lines)
        assert hits[0] > pos, (pat, lines)
        pos = hits[0]
    if len(args) >= 5 and args[4] == 3:
        assert f"\tMapping PE tile size: {args[5]} x {args[6]} rotate {args[7]} stride {args[6]} " in lines
    dg = [ln for ln in lines if ln.startswith("The dgemm")][0]
    assert f"The dgemm {args[1]} x {args[1]} takes" in dg and float(dg.split()[-2]) > 0


def test_cli_process_entry_point(cuda_dev):
    r = subprocess.run([sys.executable, "-m", "charmlu_b200", "48", "12", "500"], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = RESIDUAL.search(r.stdout)
    assert m is not None and float(m.group(1)) < 16, r.stdout


def test_cli_two_ranks_under_torchrun(cuda_dev):
    """The multi-process FP64 path (`_main_ranks`): two ranks under torchrun,
    one GPU each, print the reference's result block with residual < 16.
    Needs two GPUs; skipped otherwise."""
    import socket
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    cmd = ["timeout", "-k", "30", "600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr", "127.0.0.1", "--master-port", str(port), "-m", "charmlu_b200",
           "2048", "128", "100"]
    out = subprocess.run(cmd, capture_output=True, text=True, env=env,
                         cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out.returncode == 0, out.stderr[-2000:]
    m = RESIDUAL.search(out.stdout)
    assert m is not None, out.stdout[-2000:]
    assert float(m.group(1)) < 16
