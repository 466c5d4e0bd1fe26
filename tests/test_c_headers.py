"""The public headers compile as C (C11) and the C API links and runs from a
C program without a GPU: build a transverse-Ising operator, serialise it,
read it back."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "nutcracker.h"
#include "nutcracker_b200.h"

int main(void) {
    NutcrackerOperatorBuilder* b = Nutcracker_OperatorBuilder_newSimple(6, 2);
    double _Complex c = 0.5;
    NutcrackerMatrix* x = Nutcracker_Matrix_multiply(&c, Nutcracker_Matrix_getPauliX());
    NutcrackerOperatorTerm* t = Nutcracker_OperatorTerm_create_TransverseIsingField(
        Nutcracker_Matrix_getPauliZ(), x, Nutcracker_Matrix_getPauliX());
    Nutcracker_OperatorBuilder_addTerm(b, t);
    NutcrackerOperator* op = Nutcracker_OperatorBuilder_compile(b);
    if (!op) { printf("error %s\n", Nutcracker_getError()); return 1; }
    NutcrackerSerialization* s = Nutcracker_Operator_serialize(op);
    uint32_t n = Nutcracker_Serialization_getSize(s);
    void* buf = malloc(n);
    Nutcracker_Serialization_write(s, buf);
    NutcrackerOperator* back = Nutcracker_Operator_deserialize(n, buf);
    NutcrackerOperator* bad = Nutcracker_Operator_deserialize(3, buf);
    printf("%u %d %d %s\n", n, back != NULL, bad == NULL, Nutcracker_getError() ? "error-set" : "no-error");
    Nutcracker_Operator_free(back);
    Nutcracker_Operator_free(op);
    Nutcracker_Serialization_free(s);
    Nutcracker_OperatorTerm_free(t);
    Nutcracker_Matrix_free(x);
    Nutcracker_OperatorBuilder_free(b);
    free(buf);
    return 0;
}
"""


def test_headers_compile_as_c_and_the_c_api_runs(tmp_path):
    src = tmp_path / "prog.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "prog"
    lib = os.path.join(ROOT, "nutcracker-1_b200", "lib")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", lib, "-lnutcracker_b200", "-Wl,-rpath," + lib, "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    n, ok, bad, err = r.stdout.split()
    assert int(n) > 100 and ok == "1" and bad == "1" and err == "error-set"
