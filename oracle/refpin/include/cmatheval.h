// Test infrastructure: a project-written complex expression evaluator with
// the entry points of cmatheval that the reference's SVTensor uses.
// Expressions: + - * / ^, unary signs, parentheses, numbers, the constants
// i and pi, variables (bound by index or set to constants), and the
// functions exp, log, sqrt, sin, cos, tan, sinh, cosh, tanh, abs and step
// (0 for a negative real part, else 1).
#ifndef REFPIN_CMATHEVAL_H
#define REFPIN_CMATHEVAL_H

#include "libhrutil.h"

void *cevaluator_create(char *string);
void cevaluator_destroy(void *evaluator);
void cevaluator_set_var_index(void *evaluator, const char *name, int index);
void cevaluator_set_var(void *evaluator, const char *name, cdouble value);
cdouble cevaluator_evaluate(void *evaluator, int count, char **names, cdouble *values);

#endif
