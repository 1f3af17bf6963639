"""Drop-in replacements for the EDGE reference's util/ modules."""
