"""``CurlCurlAssemblerDiluted`` with the reference's interface
(``snoopy/curl_curl_assembler_diluted.py``).

The curl-curl assembler for magnets of diluted steel: every material may carry a
``materials.Dilution`` (or None).  A diluted material with a source field is assembled by the
diluted reduced kernel (``compute_K_dK_Hcurl_red_dil``, ``fem_c/ctools.c:1565-1759``), where the
reluctance at a quadrature point of height z is s(z) nu(s(z) |B|); every other material by
the plain or reduced kernel (``curl_curl_assembler_diluted.py:267-298``).
"""

import ctypes

import numpy as np

from . import _lib
from .curl_curl_assembler import CurlCurlAssembler
from .device import zeros


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

    def assemble_device(self, x, quad_order=2, source_fields=(), K=True, J=True, rhs=True, F=False, dK=False,
                        stream=None):
        d = self._device_state()
        tb = self.tables(quad_order)
        pat = d["pattern"]
        from .device import upload

        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        bs = self.upload_source_fields(source_fields)
        out = {"pattern": pat}
        for key, want, size in (("K", K, pat.nnz), ("J", J, pat.nnz), ("dK", dK, pat.nnz), ("rhs", rhs, self.num_dofs),
                                ("F", F, self.num_dofs)):
            out[key] = zeros(size) if want else None
        s = _lib.stream_ptr(stream)
        for n, m in enumerate(d["mats"]):
            n_int, rc, rx = d["rel"][n]
            dil = self.dilution_of(n)
            common = (pat.handle, m["offset"], m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]),
                      _lib.ptr(m["gids"]), _lib.ptr(m["orient"]), _lib.ptr(tb.curls_d), tb.n_orient)
            outs = (_lib.ptr(out["K"]), _lib.ptr(out["dK"]), _lib.ptr(out["J"]), _lib.ptr(out["rhs"]),
                    _lib.ptr(out["F"]), s)
            if dil is None:
                _lib.call("snp_curlcurl_assemble", *common, _lib.ptr(tb.d_phi_d), _lib.ptr(tb.w_d), tb.nq,
                          _lib.ptr(x_d), _lib.ptr(bs[n]), n_int, _lib.ptr(rc), _lib.ptr(rx), *outs)
            else:
                coef = (ctypes.c_double * 4)(dil.c_num, dil.m_num, dil.c_den, dil.m_den)
                _lib.call("snp_curlcurl_assemble_diluted", *common, _lib.ptr(tb.phi_d), _lib.ptr(tb.d_phi_d),
                          _lib.ptr(tb.w_d), tb.nq, _lib.ptr(x_d), _lib.ptr(bs[n]), n_int, _lib.ptr(rc), _lib.ptr(rx),
                          coef, *outs)
        return out
