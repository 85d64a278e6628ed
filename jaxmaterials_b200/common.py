"""Grid description (mirrors ``src/jaxmaterials/common.py:6-29`` of the reference)."""

__all__ = ["GridSpec"]


class GridSpec:
    """Periodic grid of nx x ny x nz voxels on a Lx x Ly x Lz box."""

    def __init__(self, nx, ny, nz, Lx, Ly, Lz):
        self.nx = int(nx)
        self.ny = int(ny)
        self.nz = int(nz)
        self.Lx = float(Lx)
        self.Ly = float(Ly)
        self.Lz = float(Lz)

    @property
    def number_of_voxels(self):
        """Return total number of voxels"""
        return self.nx * self.ny * self.nz

    @property
    def number_of_modes(self):
        """Number of modes of the real-to-complex half spectrum nx * ny * (nz/2 + 1)."""
        return self.nx * self.ny * (self.nz // 2 + 1)

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def __repr__(self):
        return (f"GridSpec({self.nx}, {self.ny}, {self.nz}, "
                f"{self.Lx}, {self.Ly}, {self.Lz})")
