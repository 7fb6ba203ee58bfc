"""The C ABI: the library loads (no GPU needed), exports every function that
include/*.h declares, and the model description has the same layout as the
oracle's (one ctypes structure drives both)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(gpgmp_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(gpgmp):
    from inchman_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_sort_scratch_size_does_not_depend_on_key_bits(gpgmp):
    """One scratch buffer serves a sort of any key width (8- and 10-bit digit layouts
    alike), so a caller may size it once for n."""
    from inchman_b200 import _lib
    L = _lib.lib()
    for n in (1, 3840, 3841, 7680, 7681, 1 << 22):
        sizes = set()
        for bits in range(1, 33):
            b = C.c_size_t(0)
            assert L.gpgmp_sort_scratch_bytes(C.c_int64(n), C.c_int32(bits), C.byref(b)) == 0
            sizes.add(b.value)
        assert len(sizes) == 1, (n, sizes)


def test_error_path_without_gpu(gpgmp):
    """Argument errors come back as codes with a message, never as a crash or exit."""
    from inchman_b200 import _lib
    L = _lib.lib()
    out = C.c_void_p()
    rc = L.gpgmp_solver_create(None, 1, 0, 0, C.byref(out))
    assert rc == 1 and b"NULL" in L.gpgmp_last_error()
    d = _lib.ModelDesc()
    d.width, d.height, d.num_species = 8, 8, 40
    rc = L.gpgmp_solver_create(C.byref(d), 1, 0, 0, C.byref(out))
    assert rc == 1 and b"num_species" in L.gpgmp_last_error()


def test_model_layout_matches_oracle():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "gpgmp_c.h"
#include "gpgmp_oracle.h"
#define P(T, f) printf("%s %zu\n", #f, offsetof(T, f))
int main(void) {
  printf("size %zu %zu %zu %zu\n", sizeof(gpgmp_model_desc), sizeof(orc_model), sizeof(gpgmp_reaction), sizeof(orc_reaction));
  P(gpgmp_model_desc, flags); P(orc_model, flags);
  P(gpgmp_model_desc, drift_params); P(orc_model, drift_params);
  P(gpgmp_model_desc, diffusion); P(orc_model, diffusion);
  P(gpgmp_model_desc, field_ry); P(orc_model, field_ry);
  P(gpgmp_model_desc, reaction_mask); P(orc_model, reaction_mask);
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"), c, "-o", exe],
                       check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = out[0].split()[1:]
    assert sizes[0] == sizes[1] and sizes[2] == sizes[3]
    pairs = [l.split() for l in out[1:] if l]
    for a, b in zip(pairs[0::2], pairs[1::2]):
        assert a[1] == b[1], (a, b)
    from inchman_b200 import _lib
    assert C.sizeof(_lib.ModelDesc) == int(sizes[0])
    assert C.sizeof(_lib.Reaction) == int(sizes[2])
