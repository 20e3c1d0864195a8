/* ORACLE - test infrastructure. Path-tracer restatement: see below. */
