"""The reference's module name for the grad-grad assembler (``snoopy/matrix_assembly.py``)."""

from .grad_grad_assembler import (GradGradAssembler, delete_cols_sparse, delete_rows_sparse,  # noqa: F401
                                  recover_full_solution)
