"""The public headers compile as C (C11) and the C API links and runs from a
C program without a GPU: build a transverse-Ising operator, serialise it,
read it back; the exported constants (Pauli matrices, qubit vectors) link
and hold the reference's values."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>
#include "nutcracker.h"
#include "nutcracker_b200.h"

int main(void) {
    NutcrackerOperatorBuilder* b = Nutcracker_OperatorBuilder_newSimple(6, 2);
    double _Complex c = 0.5;
    NutcrackerMatrix* x = Nutcracker_Matrix_multiply(&c, Nutcracker_Matrix_getPauliX());
    NutcrackerOperatorTerm* t = Nutcracker_OperatorTerm_create_TransverseIsingField(
        Nutcracker_Matrix_Pauli_Z, x, Nutcracker_Matrix_Pauli_X);
    double _Complex y01, up0, up1, dn1;
    Nutcracker_Matrix_getElementAtCoordinate(Nutcracker_Matrix_Pauli_Y, 0, 1, &y01);
    Nutcracker_Vector_getElementAtIndex(Nutcracker_Vector_Qubit_Up, 0, &up0);
    Nutcracker_Vector_getElementAtIndex(Nutcracker_Vector_Qubit_Up, 1, &up1);
    Nutcracker_Vector_getElementAtIndex(Nutcracker_Vector_Qubit_Down, 1, &dn1);
    int consts = Nutcracker_Matrix_Pauli_I == Nutcracker_Matrix_getPauliI() &&
                 Nutcracker_Matrix_Pauli_Z == Nutcracker_Matrix_getPauliZ() &&
                 y01 == -1.0 * _Complex_I && up0 == 1.0 && up1 == 0.0 && dn1 == 1.0 &&
                 Nutcracker_Vector_getSize(Nutcracker_Vector_Qubit_Down) == 2;
    Nutcracker_OperatorBuilder_addTerm(b, t);
    NutcrackerOperator* op = Nutcracker_OperatorBuilder_compile(b);
    if (!op) { printf("error %s\n", Nutcracker_getError()); return 1; }
    NutcrackerSerialization* s = Nutcracker_Operator_serialize(op);
    uint32_t n = Nutcracker_Serialization_getSize(s);
    void* buf = malloc(n);
    Nutcracker_Serialization_write(s, buf);
    NutcrackerOperator* back = Nutcracker_Operator_deserialize(n, buf);
    NutcrackerOperator* bad = Nutcracker_Operator_deserialize(3, buf);
    printf("%u %d %d %s %d\n", n, back != NULL, bad == NULL, Nutcracker_getError() ? "error-set" : "no-error",
           consts);
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
    n, ok, bad, err, consts = r.stdout.split()
    assert int(n) > 100 and ok == "1" and bad == "1" and err == "error-set" and consts == "1"
