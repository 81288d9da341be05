"""Argument checks of the drop-in CLI that precede any device use
(arguments_CUDA, L_CUDA.cu:361-410); they run without a GPU."""
import subprocess

import pytest

MSG = ("Use the following command: ./L_CUDA number_of_blocks number_of_threads_per_block "
       "filename_of_matrix order_of_the_L_norm")


def run(ld, args, cwd):
    return subprocess.run([str(ld.CLI_PATH), *args], cwd=cwd, capture_output=True, text=True,
                          timeout=60)


@pytest.fixture()
def mfile(tmp_path):
    (tmp_path / "m.txt").write_text("1 1\n1 -1\n")
    return tmp_path


@pytest.mark.parametrize("args,expect", [
    ([], f"Incorrect number of input arguments. {MSG}\n"),
    (["1", "2", "m.txt"], f"Incorrect number of input arguments. {MSG}\n"),
    (["0", "32", "m.txt", "1"], f"Please make sure that the number of blocks is a positive integer. {MSG}\n"),
    (["x", "32", "m.txt", "1"], f"Please make sure that the number of blocks is a positive integer. {MSG}\n"),
    (["8", "-1", "m.txt", "1"], f"Please make sure that the number of threads is a positive integer. {MSG}\n"),
    (["8", "4", "nope.txt", "1"], "Please make sure that the file containig the matrix exists within this directory. "
                                  f"{MSG}\n"),
    (["8", "4", "m.txt", "0"], f"Please make sure that the order of the L norm is a positive integer. {MSG}\n"),
    (["8", "4", "m.txt", "11"], "The order of the L norm is too large. Please increase the RANK_OF_NORM variable "
                                "in the code to 11 and compile and run it again.\n"),
])
def test_argument_errors(ld, mfile, args, expect):
    p = run(ld, args, mfile)
    assert p.returncode == 255
    assert p.stdout == expect
    assert not list(mfile.glob("strategy_*.txt"))
