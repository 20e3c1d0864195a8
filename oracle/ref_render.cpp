// Oracle test infrastructure (not product code). Path-tracer harness: filled in below.
