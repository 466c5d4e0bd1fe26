/* C API of the B200 library with the reference's names and argument meaning
   (includes/nutcracker.h and the sources of sources/c-interface).

   Opaque objects are created by *_new / *_compile / *_deserialize and released
   with the matching *_free.  Functions that can fail return NULL (or leave
   their outputs untouched) and set a thread-local message read with
   Nutcracker_getError() (errors.cpp).  Complex numbers are std::complex<double>
   in C++ and `double _Complex` in C (the same layout: real, imaginary).

   Operators are compiled on the host (the automaton compiler of
   compiler.hpp:419-938); solves and state contractions run on the GPU through
   the library's chain and contraction kernels. */
#ifndef NUTCRACKER_H
#define NUTCRACKER_H

#include <stdint.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> NutcrackerComplex;
extern "C" {
#else
#include <stdbool.h>
typedef double _Complex NutcrackerComplex;
#endif

typedef struct NutcrackerMatrix NutcrackerMatrix;
typedef struct NutcrackerVector NutcrackerVector;
typedef struct NutcrackerOperator NutcrackerOperator;
typedef struct NutcrackerOperatorBuilder NutcrackerOperatorBuilder;
typedef struct NutcrackerOperatorTerm NutcrackerOperatorTerm;
typedef struct NutcrackerState NutcrackerState;
typedef struct NutcrackerStateBuilder NutcrackerStateBuilder;
typedef struct NutcrackerStateTerm NutcrackerStateTerm;
typedef struct NutcrackerSerialization NutcrackerSerialization;

/* ---- errors (errors.cpp) ---- */
void Nutcracker_clearError(void);
char const* Nutcracker_getError(void);   /* NULL when no error is set */
void Nutcracker_setError(char const* message);

/* ---- square matrices (matrix.cpp); data row-major, dimension^2 entries ---- */
void Nutcracker_Matrix_free(NutcrackerMatrix* matrix);
/* includes/nutcracker.h:29-35: the Pauli matrices as exported constants,
   owned by the library (the same objects the getters below return). */
extern NutcrackerMatrix const *Nutcracker_Matrix_Pauli_I, *Nutcracker_Matrix_Pauli_X,
    *Nutcracker_Matrix_Pauli_Y, *Nutcracker_Matrix_Pauli_Z;
NutcrackerMatrix const* Nutcracker_Matrix_getPauliI(void);   /* owned by the library */
NutcrackerMatrix const* Nutcracker_Matrix_getPauliX(void);
NutcrackerMatrix const* Nutcracker_Matrix_getPauliY(void);
NutcrackerMatrix const* Nutcracker_Matrix_getPauliZ(void);
NutcrackerMatrix* Nutcracker_Matrix_new(uint32_t dimension, NutcrackerComplex const* data);
NutcrackerMatrix* Nutcracker_Matrix_newDiagonal(uint32_t dimension, NutcrackerComplex const* data);
NutcrackerMatrix* Nutcracker_Matrix_add(NutcrackerMatrix const* x, NutcrackerMatrix const* y);
NutcrackerMatrix* Nutcracker_Matrix_multiply(NutcrackerComplex const* c, NutcrackerMatrix const* x);
uint32_t Nutcracker_Matrix_getSize(NutcrackerMatrix const* x);
void Nutcracker_Matrix_getElementAtCoordinate(NutcrackerMatrix const* x, uint32_t i, uint32_t j,
                                              NutcrackerComplex* element);

/* ---- operators (operator.cpp) ---- */
void Nutcracker_Operator_free(NutcrackerOperator* op);
/* Least eigenvalues with the reference's fixed options (initial bond
   dimension 2, sanity 1e-12, site 1e-9, sweep and chain 1e-8). */
void Nutcracker_Operator_simpleSolveForLeastEigenvalues(NutcrackerOperator const* op, uint32_t number_of_levels,
                                                        float* eigenvalues);
void Nutcracker_Operator_simpleSolveForLeastEigenvaluesWithEigenvectors(NutcrackerOperator const* op,
                                                                        uint32_t number_of_levels,
                                                                        float* eigenvalues,
                                                                        NutcrackerState** eigenvectors);
NutcrackerSerialization* Nutcracker_Operator_serialize(NutcrackerOperator const* op);
NutcrackerOperator* Nutcracker_Operator_deserialize(uint32_t size, void const* buffer);

/* ---- operator builder and terms (operator_builder.cpp, operator_term.cpp) ---- */
NutcrackerOperatorBuilder* Nutcracker_OperatorBuilder_new(uint32_t number_of_sites, uint32_t* dimensions);
NutcrackerOperatorBuilder* Nutcracker_OperatorBuilder_newSimple(uint32_t number_of_sites,
                                                                uint32_t physical_dimension);
void Nutcracker_OperatorBuilder_free(NutcrackerOperatorBuilder* builder);
uint32_t Nutcracker_OperatorBuilder_numberOfSites(NutcrackerOperatorBuilder const* builder);
uint32_t Nutcracker_OperatorBuilder_dimensionOfSite(NutcrackerOperatorBuilder const* builder, uint32_t site_number);
/* components: one matrix per site; exactly number_of_sites pointers are read */
void Nutcracker_OperatorBuilder_addProductTerm(NutcrackerOperatorBuilder* builder,
                                               NutcrackerMatrix const* const* components);
void Nutcracker_OperatorBuilder_addTerm(NutcrackerOperatorBuilder* builder, NutcrackerOperatorTerm* term);
NutcrackerOperator* Nutcracker_OperatorBuilder_compile(NutcrackerOperatorBuilder* builder);
NutcrackerOperator* Nutcracker_OperatorBuilder_compileCustomized(NutcrackerOperatorBuilder* builder, bool optimize,
                                                                 bool add_start_and_end_loops);
void Nutcracker_OperatorTerm_free(NutcrackerOperatorTerm* term);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_add(NutcrackerOperatorTerm const* x, NutcrackerOperatorTerm const* y);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_multiply(NutcrackerComplex const* c, NutcrackerOperatorTerm const* x);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_LocalExternalField(uint32_t site_number,
                                                                          NutcrackerMatrix const* field_matrix);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_GlobalExternalField(NutcrackerMatrix const* field_matrix);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_LocalNeighborCouplingField(
    uint32_t site_number, NutcrackerMatrix const* left_field_matrix, NutcrackerMatrix const* right_field_matrix);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_GlobalNeighborCouplingField(
    NutcrackerMatrix const* left_field_matrix, NutcrackerMatrix const* right_field_matrix);
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_TransverseIsingField(
    NutcrackerMatrix const* external_field_matrix, NutcrackerMatrix const* left_coupling_field_matrix,
    NutcrackerMatrix const* right_coupling_field_matrix);

/* ---- serialization (serialization.cpp): the protobuf messages of
   nutcracker.proto (OperatorBuffer, StateBuffer) ---- */
void Nutcracker_Serialization_free(NutcrackerSerialization* s);
uint32_t Nutcracker_Serialization_getSize(NutcrackerSerialization* s);
void Nutcracker_Serialization_write(NutcrackerSerialization* s, void* buffer);

/* ---- states (state.cpp, state_builder.cpp, state_term.cpp) ----
   A state is a matrix product state in the reference's canonical form: the
   first site unnormalised, the others right-normalised. */
void Nutcracker_State_free(NutcrackerState* state);
void Nutcracker_State_computeOverlap(NutcrackerState const* state1, NutcrackerState const* state2,
                                     NutcrackerComplex* result);
void Nutcracker_State_computeExpectation(NutcrackerState const* state, NutcrackerOperator const* op,
                                         NutcrackerComplex* result);
NutcrackerSerialization* Nutcracker_State_serialize(NutcrackerState const* state);
NutcrackerState* Nutcracker_State_deserialize(uint32_t size, void const* buffer);
NutcrackerStateBuilder* Nutcracker_StateBuilder_new(uint32_t number_of_sites, uint32_t* dimensions);
NutcrackerStateBuilder* Nutcracker_StateBuilder_newSimple(uint32_t number_of_sites, uint32_t physical_dimension);
void Nutcracker_StateBuilder_free(NutcrackerStateBuilder* builder);
uint32_t Nutcracker_StateBuilder_numberOfSites(NutcrackerStateBuilder const* builder);
uint32_t Nutcracker_StateBuilder_dimensionOfSite(NutcrackerStateBuilder const* builder, uint32_t site_number);
void Nutcracker_StateBuilder_addProductTerm(NutcrackerStateBuilder* builder, NutcrackerVector const* const* components);
void Nutcracker_StateBuilder_addTerm(NutcrackerStateBuilder* builder, NutcrackerStateTerm* term);
NutcrackerState* Nutcracker_StateBuilder_compile(NutcrackerStateBuilder* builder);
NutcrackerState* Nutcracker_StateBuilder_compileCustomized(NutcrackerStateBuilder* builder, bool optimize);
void Nutcracker_StateTerm_free(NutcrackerStateTerm* term);
NutcrackerStateTerm* Nutcracker_StateTerm_add(NutcrackerStateTerm const* x, NutcrackerStateTerm const* y);
NutcrackerStateTerm* Nutcracker_StateTerm_multiply(NutcrackerComplex const* c, NutcrackerStateTerm const* x);
NutcrackerStateTerm* Nutcracker_StateTerm_create_ProductWithOneSiteDifferent(uint32_t site_number,
                                                                             NutcrackerVector const* common_observation,
                                                                             NutcrackerVector const* special_observation);
/* `normalized` is accepted and, as in the reference (compiler.hpp:1109-1141,
   where the flag is never stored), has no effect. */
NutcrackerStateTerm* Nutcracker_StateTerm_create_W(NutcrackerVector const* common_observation,
                                                   NutcrackerVector const* special_observation, bool normalized);

/* ---- vectors (vector.cpp) ---- */
void Nutcracker_Vector_free(NutcrackerVector* vector);
/* includes/nutcracker.h:148-151: the qubit basis vectors up = (1, 0) and
   down = (0, 1), owned by the library. */
extern NutcrackerVector const *Nutcracker_Vector_Qubit_Up, *Nutcracker_Vector_Qubit_Down;
NutcrackerVector* Nutcracker_Vector_new(uint32_t physical_dimension, NutcrackerComplex const* data);
NutcrackerVector* Nutcracker_Vector_newBasis(uint32_t physical_dimension, uint32_t observed_value);
NutcrackerVector* Nutcracker_Vector_add(NutcrackerVector const* x, NutcrackerVector const* y);
NutcrackerVector* Nutcracker_Vector_multiply(NutcrackerComplex const* c, NutcrackerVector const* x);
uint32_t Nutcracker_Vector_getSize(NutcrackerVector const* x);
void Nutcracker_Vector_getElementAtIndex(NutcrackerVector const* x, uint32_t index, NutcrackerComplex* element);

/* ---- version (version.cpp) ---- */
uint32_t Nutcracker_Version_getComponent(uint32_t index);
uint32_t Nutcracker_Version_getSize(void);
char const* Nutcracker_Version_getString(void);
void Nutcracker_Version_write(uint32_t* version);

#ifdef __cplusplus
}
#endif

#endif /* NUTCRACKER_H */
