"""The checker raises the reference's FAFERR codes 903, 904, 910 and 987 on
the data-only inputs of faferr_cases (the device tests compare the device
path's codes with these)."""
import pytest

from cpfem_code_b200 import abi

import faferr_cases


@pytest.mark.parametrize("case", sorted(faferr_cases.CASES))
def test_checker_raises(oracle_lib, case):
    from oracle import OracleSolver
    make, call, code = faferr_cases.CASES[case]
    o = OracleSolver(make(), 8, threads=4)
    with pytest.raises(abi.FasError) as ei:
        call(o)
    assert ei.value.code == code
    o.close()
