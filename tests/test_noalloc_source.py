"""The no-allocation neighbour build, checked on its source: no device allocation call appears in
it, and every call into CUB's device scan either asks for its temporary size (NULL storage) or
runs on storage inside the fixed scratch array.  (The GPU test also compares the device's free
memory around a call; the driver can serve small allocations from pages it has already mapped,
so this check covers what that comparison cannot.)"""
import os
import re

SRC = os.path.join(os.path.dirname(__file__), "..", "dmff_b200", "csrc", "noalloc.cu")


def _code():
    text = open(SRC).read()
    text = re.sub(r"//[^\n]*", "", text)
    return re.sub(r"/\*.*?\*/", "", text, flags=re.S)


def test_no_allocation_calls():
    code = _code()
    for name in ("cudaMalloc", "cudaFree", "cudaMallocAsync", "cudaFreeAsync", "cudaMallocManaged",
                 "cudaMallocHost", "cudaHostAlloc", "malloc(", "new ", "torch", "c10::", "CachingAllocator"):
        assert name not in code, name


def test_cub_calls_use_the_scratch_or_only_query_sizes():
    code = _code()
    calls = re.findall(r"cub::DeviceScan::\w+\(([^,]+),", code)
    assert len(calls) == 4
    for first in calls:
        assert first.strip() in ("nullptr", "temp"), first
    assert re.search(r"void\*\s+temp\s*=\s*\(void\*\)\(scratch\s*\+\s*kOffScanTemp\)", code)
    # the only device memory the call touches besides its arguments comes from the symbol address
    assert "cudaGetSymbolAddress" in code
