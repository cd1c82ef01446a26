"""Data-location bit helpers (N_eye of data_location_extend.f90), the same
encoding as csrc/core.cuh: bit d-1 set when the data is node-located along d."""
_BITS = {0: 0, 1: 1, 2: 2, 3: 4, 4: 6, 5: 5, 6: 3, 7: 7}
_INV = {v: k for k, v in _BITS.items()}


def dl_bits(dl: int) -> int:
    return _BITS[dl]


def dl_from_bits(b: int) -> int:
    return _INV[b]
