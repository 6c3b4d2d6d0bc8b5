"""The headers a consumer narrow phase is compiled against at upload
(sq_math.cuh and traverse.cuh, run through NVRTC by rtc.cu) must stay
compilable without the host's standard headers. This compiles the tests'
consumer sources (the near-root ball and the marched-field leaves with its
crossings hook) exactly as rtc.cu does, on the CPU: NVRTC needs no GPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "spatial_query_b200", "csrc")
NVRTC = "/usr/local/cuda/lib64/libnvrtc.so"


def consumer_source(test_file, name):
    text = open(os.path.join(ROOT, "tests", test_file)).read()
    return re.search(name + r' = """(.*?)"""', text, re.S).group(1)


def compile_rtc(src, stride, crossings):
    lib = C.CDLL(NVRTC)
    prog_src = (f"#define SQ_RTC_CUSTOM 1\n#define SQ_CUSTOM_STRIDE {stride}\n"
                + ("#define SQ_RTC_CROSSINGS 1\n" if crossings else "")
                + '#include "traverse.cuh"\nnamespace sq {\n#line 1 "narrow"\n' + src + "\n}  // namespace sq\n")
    headers = [open(os.path.join(CSRC, h)).read().encode() for h in ("sq_math.cuh", "traverse.cuh")]
    hdr = (C.c_char_p * 2)(*headers)
    names = (C.c_char_p * 2)(b"sq_math.cuh", b"traverse.cuh")
    prog = C.c_void_p()
    assert lib.nvrtcCreateProgram(C.byref(prog), prog_src.encode(), b"consumer_narrow.cu", 2, hdr, names) == 0
    for k in (b"&sq::query_kernel<3, 4, 0, false, false, false>", b"&sq::query_kernel<3, 4, 1, true, false, false>"):
        lib.nvrtcAddNameExpression(prog, k)
    opts = (C.c_char_p * 4)(b"--gpu-architecture=sm_100a", b"-std=c++17", b"--fmad=false", b"-diag-suppress=549")
    rc = lib.nvrtcCompileProgram(prog, 4, opts)
    n = C.c_size_t(0)
    lib.nvrtcGetProgramLogSize(prog, C.byref(n))
    log = C.create_string_buffer(n.value + 1)
    lib.nvrtcGetProgramLog(prog, log)
    lib.nvrtcDestroyProgram(C.byref(prog))
    return rc, log.value.decode(errors="replace")


@pytest.mark.skipif(not os.path.exists(NVRTC), reason="NVRTC is not installed")
@pytest.mark.parametrize("test_file,name,stride,crossings", [
    ("test_gpu_custom_narrow.py", "BALL_NEAR", 4, False),
    ("test_gpu_field.py", "FIELD", 6, True),
])
def test_consumer_source_compiles(test_file, name, stride, crossings):
    rc, log = compile_rtc(consumer_source(test_file, name), stride, crossings)
    assert rc == 0, log
