"""FP64 host oracle (test infrastructure only; the product never imports it)."""
