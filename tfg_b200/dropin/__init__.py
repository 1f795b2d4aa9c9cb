"""The reference-side binding: the reference's host entry points over the C ABI (see reference_wrappers.cu)."""
