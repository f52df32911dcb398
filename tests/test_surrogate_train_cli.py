"""The training command's sample-count parser (no GPU)."""
from openstc_b200.surrogate_train import count


def test_count_suffixes():
    assert count("16M") == 16 * (1 << 20)
    assert count("1m") == 1 << 20
    assert count("512K") == 512 * 1024
    assert count("1000") == 1000
    assert count("0.5M") == 1 << 19
