"""Python cffi binding of libd3.so, API-compatible with LASP-D3's src/d3_cffi.py.

Same module-level `ffi` / `lib` objects and the same `D3Calculator` class with the same
constructor defaults, methods and return values (energy as float, forces float32
[n, 3], stress float32 [3, 3]; status 0b01 raises "neighbor list overflow",
src/d3_cffi.py:96-120). Additions, all optional:
  * `init_d3_handle_with_atm` is declared, and D3Calculator takes `atm_cutoff`
    (bohr) to enable the ATM three-body term (the reference's binding cannot reach it,
    src/d3_cffi.py:8-45 omits the declaration);
  * `compute_f64()` returns the FP64 results of the same evaluation path;
  * `D3BatchCalculator` evaluates many independent periodic structures in one call
    (d3_init_batch / d3_set_batch_f64 / d3_compute_batch_f64);
  * the library path can be overridden with the D3_LIBRARY environment variable.
"""
import os

import cffi
import numpy as np

ffi = cffi.FFI()

ffi.cdef("""
typedef void d3_handle_t;

void compute_dispersion_energy(
    float atoms[][3],
    uint16_t *elements,
    uint64_t num_atoms,
    float cell[3][3],
    float cutoff_radius,
    float CN_cutoff_radius,
    int damping_type,
    int functional_type,
    float *energy,
    float *force,
    float *stress
);

d3_handle_t *init_d3_handle(
    uint16_t *elements,
    uint64_t length_elements,
    uint64_t max_length,
    float cutoff_radius,
    float coordination_number_cutoff,
    int damping_type,
    int functional_type
);

d3_handle_t *init_d3_handle_with_atm(
    uint16_t *elements,
    uint64_t length_elements,
    uint64_t max_length,
    float cutoff_radius,
    float coordination_number_cutoff,
    float atm_cutoff,
    int damping_type,
    int functional_type
);

void set_atoms(d3_handle_t *handle, float *coords, uint16_t *elements, uint64_t length);
void set_cell(d3_handle_t *handle, float cell[3][3]);
void free_d3_handle(d3_handle_t *handle);
void clear_d3_handle(d3_handle_t *handle);
uint16_t compute_dispersion_energy_from_handle_status(
    d3_handle_t *handle,
    float *energy,
    float *force,
    float *stress
);

uint16_t d3_compute_f64(d3_handle_t *handle, double *energy, double *force, double *stress);
const char *d3_last_error(void);

d3_handle_t *d3_init_batch(const uint16_t *elements, uint64_t n_elements, uint64_t max_structures,
                           uint64_t max_total_atoms, double rc, double rc_cn, double rc_atm, int damping_type,
                           int functional_type, int table);
int d3_set_batch_f64(d3_handle_t *handle, uint64_t n_structures, const uint64_t *atom_counts, const double *coords,
                     const uint16_t *elements, const double *cells);
uint16_t d3_compute_batch_f64(d3_handle_t *handle, double *energies, double *forces, double *stresses);
int d3_num_structures(d3_handle_t *handle);
""")

lib_path = os.environ.get("D3_LIBRARY") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libd3.so")
lib = ffi.dlopen(lib_path)


class D3Calculator:
    def __init__(self, elements: list[int], max_length: int, cutoff_radius: float = 46.475800,
                 cn_cutoff_radius: float = 46.475800, damping_type: int = 0, functional_type: int = 0,
                 atm_cutoff: float | None = None):
        """Initialize a D3 calculator object (atm_cutoff in bohr enables ATM)."""
        elements_array = np.array(elements, dtype=np.uint16)
        elements_ptr = ffi.cast("uint16_t*", elements_array.ctypes.data)
        if atm_cutoff is None:
            self.handle = lib.init_d3_handle(elements_ptr, len(elements_array), max_length, cutoff_radius,
                                             cn_cutoff_radius, damping_type, functional_type)
        else:
            self.handle = lib.init_d3_handle_with_atm(elements_ptr, len(elements_array), max_length, cutoff_radius,
                                                      cn_cutoff_radius, atm_cutoff, damping_type, functional_type)
        if self.handle == ffi.NULL:
            raise RuntimeError("failed to initialise the D3 handle: " + ffi.string(lib.d3_last_error()).decode())
        self.num_atoms = max_length

    def set_atoms(self, coords: np.ndarray, elements: list[int]):
        """Set atom coordinates (Angstrom) and elements."""
        coords_array = np.ascontiguousarray(coords, dtype=np.float32)
        elements_array = np.ascontiguousarray(elements, dtype=np.uint16)
        coords_ptr = ffi.cast("float*", coords_array.ctypes.data)
        elements_ptr = ffi.cast("uint16_t*", elements_array.ctypes.data)
        lib.set_atoms(self.handle, coords_ptr, elements_ptr, len(elements_array))
        self.num_atoms = len(elements_array)

    def set_cell(self, cell: np.ndarray):
        """Set the periodic cell (Angstrom, rows are lattice vectors)."""
        cell_array = np.ascontiguousarray(cell, dtype=np.float32)
        cell_ptr = ffi.cast("float (*)[3]", cell_array.ctypes.data)
        lib.set_cell(self.handle, cell_ptr)

    def compute(self):
        """Compute dispersion energy (eV), forces (eV/A) and stress (eV/A^3)."""
        num_atoms = self.num_atoms
        if num_atoms <= 0:
            raise ValueError("Number of atoms must be greater than zero.")
        energy = ffi.new("float*")
        forces = np.zeros((num_atoms, 3), dtype=np.float32)
        stress = np.zeros(9, dtype=np.float32)
        forces_ptr = ffi.cast("float*", forces.ctypes.data)
        stress_ptr = ffi.cast("float*", stress.ctypes.data)
        result = lib.compute_dispersion_energy_from_handle_status(self.handle, energy, forces_ptr, stress_ptr)
        if result == 0b01:
            raise RuntimeError("Error computing dispersion energy: neighbor list overflow")
        return float(energy[0]), forces, stress.reshape(3, 3)

    def compute_f64(self):
        """FP64 results of the same evaluation: (energy, forces [n,3], stress [3,3])."""
        energy = ffi.new("double*")
        forces = np.zeros((self.num_atoms, 3), dtype=np.float64)
        stress = np.zeros(9, dtype=np.float64)
        result = lib.d3_compute_f64(self.handle, energy, ffi.cast("double*", forces.ctypes.data),
                                    ffi.cast("double*", stress.ctypes.data))
        if result == 0b01:
            raise RuntimeError("Error computing dispersion energy: neighbor list overflow")
        return float(energy[0]), forces, stress.reshape(3, 3)

    def clear(self):
        """Clear the D3 handle data."""
        lib.clear_d3_handle(self.handle)

    def __del__(self):
        """Clean up when the object is deleted."""
        if hasattr(self, "handle") and self.handle != ffi.NULL:
            lib.free_d3_handle(self.handle)
            self.handle = ffi.NULL


class D3BatchCalculator:
    """Many independent periodic structures in one handle, FP64 in and out (cutoffs in
    bohr, atm_cutoff None disables ATM)."""

    def __init__(self, elements: list[int], max_structures: int, max_total_atoms: int, cutoff_radius: float = 95.0,
                 cn_cutoff_radius: float = 40.0, atm_cutoff: float | None = None, damping_type: int = 1,
                 functional_type: int = 0, table: int = 0):
        el = np.array(sorted(set(int(z) for z in elements)), dtype=np.uint16)
        self._el = el
        self.handle = lib.d3_init_batch(ffi.cast("uint16_t*", el.ctypes.data), len(el), max_structures,
                                        max_total_atoms, cutoff_radius, cn_cutoff_radius, atm_cutoff or 0.0,
                                        damping_type, functional_type, table)
        if self.handle == ffi.NULL:
            raise RuntimeError("failed to initialise the D3 batch handle: " + ffi.string(lib.d3_last_error()).decode())
        self.counts = None

    def set_structures(self, structures):
        """structures: sequence of (coords [n, 3] Angstrom, elements [n], cell [3, 3] Angstrom)."""
        counts = np.array([len(z) for _, z, _ in structures], dtype=np.uint64)
        coords = np.ascontiguousarray(np.concatenate([np.asarray(c, np.float64) for c, _, _ in structures]))
        z = np.ascontiguousarray(np.concatenate([np.asarray(e, np.uint16) for _, e, _ in structures]))
        cells = np.ascontiguousarray(np.stack([np.asarray(c, np.float64).reshape(9) for _, _, c in structures]))
        if lib.d3_set_batch_f64(self.handle, len(counts), ffi.cast("uint64_t*", counts.ctypes.data),
                                ffi.cast("double*", coords.ctypes.data), ffi.cast("uint16_t*", z.ctypes.data),
                                ffi.cast("double*", cells.ctypes.data)):
            raise RuntimeError(ffi.string(lib.d3_last_error()).decode())
        self.counts = counts

    def compute(self):
        """Energies [S] (eV), forces per structure [n_s, 3] (eV/A), stresses [S, 3, 3] (eV/A^3)."""
        S, n = len(self.counts), int(self.counts.sum())
        e = np.zeros(S)
        f = np.zeros((n, 3))
        st = np.zeros((S, 9))
        result = lib.d3_compute_batch_f64(self.handle, ffi.cast("double*", e.ctypes.data),
                                          ffi.cast("double*", f.ctypes.data), ffi.cast("double*", st.ctypes.data))
        if result == 0b01:
            raise RuntimeError("Error computing dispersion energy: neighbor list overflow")
        if result:
            raise RuntimeError("d3_compute_batch_f64 status %d: %s" % (result, ffi.string(lib.d3_last_error()).decode()))
        off = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        return e, [f[off[k]:off[k + 1]] for k in range(S)], st.reshape(S, 3, 3)

    def __del__(self):
        if hasattr(self, "handle") and self.handle != ffi.NULL:
            lib.free_d3_handle(self.handle)
            self.handle = ffi.NULL
