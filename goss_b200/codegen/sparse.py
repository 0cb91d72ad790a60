"""Structure-aware Newton linear algebra for the implicit solvers' kernels.

The reference factorises ``I - h*alpha*J`` with a dense Doolittle LU without
pivoting (``ODE::lu_factorize``, ``cpp/goss/ODE.cpp:69-100``) and solves with
``ODE::forward_backward_subst`` (``ODE.cpp:102-132``).  For cell models the
Jacobian is mostly structural zeros: a gating variable's rate depends on the
membrane potential and on itself only, so TT04's 17x17 Jacobian has 67
non-zeros and 71 after the fill-in of the LU in natural order (45 multiply-adds
instead of ~4,900).

The generated code below runs the reference's loops in the reference's order
but drops every product one of whose factors stays structurally zero through
the factorisation.  Such a product is exactly 0 (a forward-difference entry
outside the structure is ``(f - f)/delta``, an analytic one is the constant
0), and adding an exact 0 to a finite sum leaves it unchanged, so for finite
matrices the factors and solutions are bit-identical to the dense loops.  The
matrix is stored packed: entry (r, c) of the LU structure at position
``pos[(r, c)]`` (row-major over the structure).
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple


class LUStructure:
    """Symbolic Doolittle factorisation of an n x n structure (diagonal added)."""

    def __init__(self, jac_structure: Sequence[Sequence[bool]]):
        n = len(jac_structure)
        self.n = n
        self.jac = [[bool(v) for v in row] for row in jac_structure]
        A = [row[:] for row in self.jac]
        for i in range(n):
            A[i][i] = True
        # fill-in of Gaussian elimination in natural order (= Doolittle's)
        for k in range(n):
            for i in range(k + 1, n):
                if A[i][k]:
                    for j in range(k + 1, n):
                        if A[k][j]:
                            A[i][j] = True
        self.lu = A
        self.pos: Dict[Tuple[int, int], int] = {}
        for r in range(n):
            for c in range(n):
                if A[r][c]:
                    self.pos[(r, c)] = len(self.pos)
        self.nnz = len(self.pos)
        self.diag = [self.pos[(i, i)] for i in range(n)]
        # positions in the LU structure that are not Jacobian entries (set to 0
        # before a forward-difference Jacobian fills the others)
        self.extra = [p for (r, c), p in self.pos.items() if not self.jac[r][c]]

    def nz(self, r: int, c: int) -> bool:
        return self.lu[r][c]

    # -- generated bodies (``J`` an indexable of doubles, packed) ------------
    def _dot(self, pairs: List[Tuple[int, int]], J: str) -> List[str]:
        out = ["double s = 0.0;"]
        for a, b in pairs:
            out.append(f"s = s + {J}[{a}] * {J}[{b}];")
        return out

    def lu_factorize_lines(self, J: str = "J") -> List[str]:
        """In-place Doolittle LU (``ODE::lu_factorize``'s loop order)."""
        n, p, nz = self.n, self.pos, self.nz
        L: List[str] = []
        for k in range(1, n):
            for i in range(k):
                if nz(i, k):
                    pairs = [(p[(i, r)], p[(r, k)]) for r in range(i) if nz(i, r) and nz(r, k)]
                    if pairs:
                        L.append("{ " + " ".join(self._dot(pairs, J)) + f" {J}[{p[(i, k)]}] -= s; }}")
                if nz(k, i):
                    pairs = [(p[(k, r)], p[(r, i)]) for r in range(i) if nz(k, r) and nz(r, i)]
                    dot = " ".join(self._dot(pairs, J)) if pairs else "const double s = 0.0;"
                    L.append("{ " + dot + f" {J}[{p[(k, i)]}] = ({J}[{p[(k, i)]}] - s) / {J}[{p[(i, i)]}]; }}")
            pairs = [(p[(k, r)], p[(r, k)]) for r in range(k) if nz(k, r) and nz(r, k)]
            if pairs:
                L.append("{ " + " ".join(self._dot(pairs, J)) + f" {J}[{p[(k, k)]}] -= s; }}")
        return L

    def solve_lines(self, J: str = "J", b: str = "b", x: str = "x") -> List[str]:
        """Forward then backward substitution (``ODE::forward_backward_subst``);
        ``b`` and ``x`` may be the same array."""
        n, p, nz = self.n, self.pos, self.nz
        L = [f"{x}[0] = {b}[0];"]
        for i in range(1, n):
            terms = [(p[(i, j)], j) for j in range(i) if nz(i, j)]
            if terms:
                body = " ".join(f"s = s + {J}[{a}] * {x}[{j}];" for a, j in terms)
                L.append(f"{{ double s = 0.0; {body} {x}[{i}] = {b}[{i}] - s; }}")
            else:
                L.append(f"{x}[{i}] = {b}[{i}] - 0.0;")
        L.append(f"{x}[{n - 1}] = {x}[{n - 1}] / {J}[{p[(n - 1, n - 1)]}];")
        for i in range(n - 2, -1, -1):
            terms = [(p[(i, j)], j) for j in range(i + 1, n) if nz(i, j)]
            body = " ".join(f"s = s + {J}[{a}] * {x}[{j}];" for a, j in terms)
            L.append(f"{{ double s = 0.0; {body} {x}[{i}] = ({x}[{i}] - s) / {J}[{p[(i, i)]}]; }}")
        return L

    def shift_lines(self, J: str = "J", scale: str = "scale") -> List[str]:
        """``J := scale*J + I`` in the reference's two passes
        (``ImplicitODESolver.cpp:99-100``: ``mult`` then ``add_mass_matrix``)."""
        L = [f"for (int k = 0; k < {self.nnz}; ++k) {J}[k] = {J}[k] * {scale};"]
        L += [f"{J}[{d}] = {J}[{d}] + 1.0 * 1.0;" for d in self.diag]
        return L

    def copy_shift_lines(self, src: str, dst: str, scale: str) -> List[str]:
        """``dst := scale*src + I`` (ESDIRK23a keeps the Jacobian and its
        factorisation apart, ``ESDIRK23a.cpp:101-115``)."""
        L = [f"for (int k = 0; k < {self.nnz}; ++k) {dst}[k] = {src}[k] * {scale};"]
        L += [f"{dst}[{d}] = {dst}[{d}] + 1.0 * 1.0;" for d in self.diag]
        return L

    def fd_column_lines(self, J: str = "J") -> List[str]:
        """``switch`` over column i storing ``(f2[r] - f1[r]) / delta`` at the
        structural rows of that column."""
        n, p = self.n, self.pos
        L = ["switch (i) {"]
        for c in range(n):
            rows = [r for r in range(n) if self.jac[r][c]]
            stores = " ".join(f"{J}[{p[(r, c)]}] = (f2[{r}] - f1[{r}]) / delta;" for r in rows)
            L.append(f"case {c}: {stores} break;")
        L.append("default: break;")
        L.append("}")
        return L

    def clear_extra_lines(self, J: str = "J") -> List[str]:
        return [f"{J}[{k}] = 0.0;" for k in self.extra]
