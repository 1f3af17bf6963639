"""Drop-in replacements for the EDGE reference's sim/ modules (same names and
arguments; fields are torch CUDA tensors in the reference's layout)."""
