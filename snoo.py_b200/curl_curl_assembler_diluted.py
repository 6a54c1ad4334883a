"""``CurlCurlAssemblerDiluted`` with the reference's interface
(``snoopy/curl_curl_assembler_diluted.py``).

The curl-curl assembler for magnets of diluted steel: every material may carry a
``materials.Dilution`` (or None).  A diluted material with a source field is assembled by the
diluted reduced kernel (``compute_K_dK_Hcurl_red_dil``, ``fem_c/ctools.c:1565-1759``), where the
reluctance at a quadrature point of height z is s(z) nu(s(z) |B|); every other material by
the plain or reduced kernel (``curl_curl_assembler_diluted.py:267-298``).
"""

import ctypes

from .curl_curl_assembler import CurlCurlAssembler


class CurlCurlAssemblerDiluted(CurlCurlAssembler):
    """Assembler of the Newton system with diluted iron (``curl_curl_assembler_diluted.py:17``).

    :param dilutions_list: one ``Dilution`` or None per entry of ``material_list``.
    """

    def __init__(self, mesh, volume_tags, material_list, dilutions_list, element_order=1):
        super().__init__(mesh, volume_tags, material_list, element_order)
        self.dilutions = list(dilutions_list)

    def dilution_of(self, n):
        """The Dilution of material ``n`` (None when the material is plain iron or air)."""
        return self.dilutions[n] if n < len(self.dilutions) else None

    def _dilution_coef(self, n):
        dil = self.dilution_of(n)
        if dil is None:
            return None
        return (ctypes.c_double * 4)(dil.c_num, dil.m_num, dil.c_den, dil.m_den)
