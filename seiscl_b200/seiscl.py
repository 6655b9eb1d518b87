"""SeisCL-compatible Python front end over the CUDA engine.

The class mirrors the public interface of ``SeisCL/SeisCL.py`` (class
``SeisCL``, SeisCL.py:33-1085): the same constructor keywords and defaults,
the same attribute names (the reference calls them ``csts``), the same
``set_forward`` / ``set_backward`` / ``execute`` / ``read_*`` sequence and the
same array orientations (models ``N``-shaped, seismograms ``NT x ntraces``,
``src_pos_all`` 5 x nsrc, ``rec_pos_all`` 8 x ntraces).

The reference writes HDF5 files into ``workdir`` and runs the
``SeisCL_MPI`` executable, which reads them back (SeisCL.py:459-505,
src/read_hdf5.c, src/writehdf5.c).  Here ``execute`` drives the time loop of
src/time_stepping.c:693-900 in-process through the C ABI of
``libseiscl_b200.so`` on the current CUDA device, and the job files are
records keyed by the same file names: kept in memory by default, or -- with
``files=True`` -- written to and read from HDF5 files in ``workdir`` with the
reference's names, datasets and transposes (``seiscl_b200.h5lite``), so a
workflow that exchanges files, or the command line
``python -m seiscl_b200.cli <base> [din]`` (SeisCL_MPI's arguments), works on
the same files:

* per shot (sources grouped by ascending ``srcid``, read_hdf5.c:357-393):
  forward modelling with the selected seismogram outputs;
* when observed data are present and gradients, residuals or the misfit are
  requested: the L2 residual of src/residuals.c:58-450 (optional Butterworth
  band-pass, trace/shot rms scaling), the residual scaling of
  residuals.c:452 (``res_scale``), the boundary-saving adjoint and the
  gradient accumulation;
* after the last shot: the parameter chain rule of src/calc_grad.c
  (``transf_grad``) and the misfit ``rms``/``rms_norm`` of writehdf5.c:249-257.

The engine is the only compute path: if ``libseiscl_b200.so`` cannot be
loaded the constructor raises ``SeisCLError``, as the reference does when no
SeisCL executable is found (SeisCL.py:268-285).
"""
from __future__ import annotations

import os
import time
from typing import Dict, List, Optional

import numpy as np

from . import engine
from . import h5lite
from . import shots as shots_mod

# The keys SeisCL writes to and reads from the constants file (SeisCL.py:23-30)
CSTS = ['N', 'ND', 'dh', 'dt', 'NT', 'freesurf', 'FDORDER', 'MAXRELERROR',
        'L', 'f0', 'FL', 'src_pos', 'rec_pos', 'src', 'abs_type', 'VPPML',
        'NPOWER', 'FPML', 'K_MAX_CPML', 'nab', 'abpc', 'pref_device_type',
        'no_use_GPUs', 'MPI_NPROC_SHOT', 'nmax_dev', 'back_prop_type',
        'param_type', 'gradfreqs', 'tmax', 'tmin', 'scalerms',
        'scalermsnorm', 'scaleshot',
        'fmin', 'fmax', 'gradout', 'Hout', 'gradsrcout', 'seisout', 'resout',
        'rmsout', 'movout', 'restype', 'inputres', 'FP16']


def _to_file(name: str, value):
    """An in-memory record value as its HDF5 dataset: SeisCL.py writes
    np.transpose(array) (N-shaped models become [nx][(ny)][nz] z-fastest, NT x
    ntraces seismograms [ntraces][NT]); movies are kept in file order."""
    a = np.asarray(value)
    return a if name.startswith("mov") else np.transpose(a)


def _from_file(name: str, value):
    a = np.asarray(value)
    return a if name.startswith("mov") else np.transpose(a)

# Seismogram variables of each modelling case (assign_modeling_case.c:1242-1322);
# "p" is a transformed variable of the elastic cases and a field in acoustics.
_VARS = {
    2: ["vx", "vz", "sxx", "szz", "sxz", "p"],
    3: ["vx", "vy", "vz", "sxx", "syy", "szz", "sxz", "sxy", "syz", "p"],
    21: ["vy", "sxy", "syz"],
    22: ["vx", "vz", "p"],
}


class SeisCLError(Exception):
    """Raised for every user-facing failure, as SeisCL.py:20-30."""


def next_fast_size(n: int) -> int:
    """Smallest m >= n whose only prime factors are 2, 3 and 5.

    The FFT length rule of kiss_fft_next_fast_size, used by the band-pass
    filter of src/butterworth.c:31."""
    m = max(int(n), 1)
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def butterworth(data: np.ndarray, fcl: float, fch: float, dt: float, tmax: int, order: int = 6) -> np.ndarray:
    """Zero-phase Butterworth amplitude filter of src/butterworth.c:25-86.

    ``data`` is [ntrace][NT]; the first ``tmax`` samples of each trace are
    filtered in place (a copy is returned). The trace is padded to the next
    2-3-5 FFT length by repeating its own first samples, multiplied in the
    frequency domain by the high-pass ``1 - sqrt(1/(1+(f/fcl)^(2n)))`` and
    low-pass ``sqrt(1/(1+(f/fch)^(2n)))`` responses, and transformed back."""
    out = np.array(data, dtype=np.float32, copy=True)
    nfft = next_fast_size(tmax)
    freq = np.arange(nfft // 2 + 1) / (dt * nfft)
    H = np.ones(nfft // 2 + 1)
    if fcl > 0:
        H *= 1.0 - np.sqrt(1.0 / (1.0 + (freq / fcl) ** (2 * order)))
    if fch > 0:
        H *= np.sqrt(1.0 / (1.0 + (freq / fch) ** (2 * order)))
    buf = np.empty((out.shape[0], nfft), np.float64)
    buf[:, :tmax] = out[:, :tmax]
    buf[:, tmax:] = out[:, : nfft - tmax]
    spec = np.fft.rfft(buf, axis=1) * H
    out[:, :tmax] = np.fft.irfft(spec, n=nfft, axis=1)[:, :tmax]
    return out


class SeisCL:
    """Drop-in counterpart of ``SeisCL.SeisCL`` running on the CUDA engine."""

    def __init__(self,
                 N: np.ndarray = None, ND: int = 2, dh: float = 10,
                 dt: float = 0.0008, NT: int = 875,
                 L: int = 0, f0: float = 15, FL: np.ndarray = np.array(15),
                 FDORDER: int = 8, MAXRELERROR: int = 1, FP16: int = 0,
                 src_pos_all: np.ndarray = np.empty((5, 0)),
                 rec_pos_all: np.ndarray = np.empty((8, 0)),
                 src_all: np.ndarray = None,
                 freesurf: int = 0, abs_type: int = 1,
                 VPPML: float = 3500, NPOWER: float = 2, FPML: float = 15,
                 K_MAX_CPML: float = 2, nab: int = 16, abpc: float = 6,
                 with_docker: bool = False, with_mpi: bool = False,
                 NP: int = 1, pref_device_type: int = 4,
                 MPI_NPROC_SHOT: int = 1, nmax_dev: int = 1,
                 no_use_GPUs: np.ndarray = np.array([-1]),
                 gradout: int = 0, Hout: int = 0, gradsrcout: int = 0,
                 back_prop_type: int = 1, cropgrad=True,
                 gradfreqs: np.ndarray = np.empty((1, 0)), param_type: int = 0,
                 tmax: float = 0, tmin: float = 0, fmin: float = 0,
                 fmax: float = 0, filter_offset: bool = False,
                 offmin: float = -float('Inf'), offmax: float = float('Inf'),
                 inputres: int = 0, restype: int = 0, scalerms: int = 0,
                 scalermsnorm: int = 0, scaleshot: int = 0,
                 seisout: int = 2, resout: int = 0, rmsout: int = 0,
                 movout: int = 0,
                 file: str = "SeisCL", workdir: str = "./seiscl",
                 files: bool = False,
                 ):
        """Keyword meanings and defaults are those of SeisCL.py:38-300.

        Accepted for compatibility but without effect on a single CUDA
        device: ``with_docker``, ``with_mpi``, ``NP``, ``pref_device_type``,
        ``MPI_NPROC_SHOT``, ``nmax_dev``, ``no_use_GPUs`` (shots are spread
        over ranks by ``seiscl_b200.shots`` instead). ``FP16`` 2 or 3 stores
        the saved boundaries in FP16 and, for forward runs of 3D and 2D P-SV
        grids with L <= 3, the wave fields and memory variables too
        (power-of-two scaled, as the reference's FP16=2 mode); arithmetic is
        FP32 in every mode.

        ``files`` (no counterpart in the reference, which always uses files):
        True writes and reads the job files as HDF5 in ``workdir``; False
        keeps them in memory."""
        try:
            engine.load_library()
        except Exception as exc:  # the engine is the only compute path
            raise SeisCLError("No working SeisCL engine found: %s" % exc) from exc

        self.N = N
        self.ND = ND
        self.dh = dh
        self.dt = dt
        self.NT = NT
        self.L = L
        self.f0 = f0
        self.FL = FL
        self.FDORDER = FDORDER
        self.MAXRELERROR = MAXRELERROR
        self.FP16 = FP16
        self.src_pos_all = src_pos_all
        self.rec_pos_all = rec_pos_all
        self.src_all = src_all
        self.src_pos = None
        self.rec_pos = None
        self.src = None
        self.freesurf = freesurf
        self.abs_type = abs_type
        self.VPPML = VPPML
        self.NPOWER = NPOWER
        self.FPML = FPML
        self.K_MAX_CPML = K_MAX_CPML
        self.nab = nab
        self.abpc = abpc
        self.with_docker = with_docker
        self.with_mpi = with_mpi
        self.NP = NP
        self.pref_device_type = pref_device_type
        self.MPI_NPROC_SHOT = MPI_NPROC_SHOT
        self.nmax_dev = nmax_dev
        self.no_use_GPUs = no_use_GPUs
        self.gradout = gradout
        self.Hout = Hout
        self.gradsrcout = gradsrcout
        self.back_prop_type = back_prop_type
        self.cropgrad = cropgrad
        self.gradfreqs = gradfreqs
        self.param_type = param_type
        self.tmax = tmax
        self.tmin = tmin
        self.fmin = fmin
        self.fmax = fmax
        self.filter_offset = filter_offset
        self.offmin = offmin
        self.offmax = offmax
        self.inputres = inputres
        self.restype = restype
        self.scalerms = scalerms
        self.scalermsnorm = scalermsnorm
        self.scaleshot = scaleshot
        self.seisout = seisout
        self.resout = resout
        self.rmsout = rmsout
        self.movout = movout
        self.progname = "libseiscl_b200"
        self.file = file
        self.file_datalist = None
        self.workdir = workdir
        self.wavelet_generator = self.ricker_wavelet
        self.__to_load_names = None
        # The job files, keyed by file name (also written to / read from
        # workdir as HDF5 when use_files)
        self.use_files = bool(files)
        self._files: Dict[str, Dict[str, np.ndarray]] = {}
        self._model: Optional[Dict[str, np.ndarray]] = None
        self._plan = None
        self._plan_key = None

    # ------------------------------------------------------------ properties
    @property
    def workdir(self):
        return self.__workdir

    @workdir.setter
    def workdir(self, workdir):
        self.__workdir = workdir

    @property
    def file_datalist(self):
        return self.__file_datalist

    @file_datalist.setter
    def file_datalist(self, file_datalist):
        """A data list holds src_pos, rec_pos and src (SeisCL.py:327-336); here
        it is an ``.npz`` file with the reference's (transposed) layout."""
        self.__file_datalist = file_datalist
        if file_datalist:
            with np.load(file_datalist) as mat:
                for word, attr in (("src_pos", "src_pos_all"), ("rec_pos", "rec_pos_all"), ("src", "src_all")):
                    setattr(self, attr, np.transpose(mat[word]))

    @property
    def params(self):
        """Parameter names of the chosen parametrisation (SeisCL.py:340-354)."""
        if self.param_type == 0:
            params = ['vp', 'vs', 'rho']
        elif self.param_type == 1:
            params = ['M', 'mu', 'rho']
        elif self.param_type == 2:
            params = ['Ip', 'Is', 'rho']
        else:
            raise NotImplementedError()
        if self.L > 0:
            params.append('taup')
            params.append('taus')
        return params

    @property
    def file(self):
        return self.__file

    @file.setter
    def file(self, file):
        self.__file = file
        self.file_model = file + "_model.mat"
        self.file_csts = file + "_csts.mat"
        self.file_dout = file + "_dout.mat"
        self.file_gout = file + "_gout.mat"
        self.file_rms = file + "_rms.mat"
        self.file_movout = file + "_movie.mat"
        self.file_din = file + "_din.mat"
        self.file_res = file + "_res.mat"

    @property
    def csts(self):
        return self.__dict__

    # ------------------------------------------------------------ job files
    def _path(self, filename, workdir=None):
        if os.path.isabs(filename):
            return filename
        return os.path.join(self.workdir if workdir is None else workdir, filename)

    def _put(self, filename, record, workdir=None):
        """Store a job file: in memory, and as HDF5 in workdir when use_files."""
        self._files[os.path.basename(filename)] = record
        if self.use_files:
            path = self._path(filename, workdir)
            os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
            try:
                h5lite.write(path, {k: _to_file(k, v) for k, v in record.items()
                                    if v is not None and np.asarray(v).dtype.kind in "biuf"})
            except (OSError, h5lite.H5Error) as exc:
                raise SeisCLError("could not write %s: %s\n" % (path, exc)) from exc

    def _get(self, filename, workdir=None):
        """A job file's record, or None when there is none."""
        if self.use_files:
            path = self._path(filename, workdir)
            if not os.path.exists(path):
                return None
            try:
                return {k: _from_file(k, v) for k, v in h5lite.read(path).items()}
            except (OSError, h5lite.H5Error) as exc:
                raise SeisCLError("could not read %s: %s\n" % (path, exc)) from exc
        return self._files.get(os.path.basename(filename))

    @property
    def to_load_names(self):
        """Seismogram names for ``seisout`` (SeisCL.py:377-409); the acoustic
        case (ND=22) outputs vx, vz and p as in assign_modeling_case.c."""
        if self.__to_load_names is not None:
            return self.__to_load_names
        nd = self.ND
        if self.seisout == 1:
            return {2: ["vx", "vz"], 21: ["vy"], 3: ["vx", "vy", "vz"], 22: ["vx", "vz"]}.get(nd)
        if self.seisout == 2:
            return ["p"]
        if self.seisout == 3:
            return {2: ["sxx", "szz", "sxz"], 21: ["sxy", "syz"],
                    3: ["sxx", "syy", "szz", "sxz", "sxy", "syz"], 22: ["p"]}.get(nd)
        if self.seisout == 4:
            return {2: ["vx", "vz", "sxx", "szz", "sxz"], 21: ["vy", "sxy", "syz"],
                    3: ["vx", "vy", "vz", "sxx", "syy", "szz", "sxz", "sxy", "syz"],
                    22: ["vx", "vz", "p"]}.get(nd)
        return None

    @to_load_names.setter
    def to_load_names(self, values):
        self.__to_load_names = values

    # ---------------------------------------------------------- job set-up
    def set_forward(self, jobids, params, workdir=None, withgrad=True):
        """Select the shots and the model of the next ``execute`` (SeisCL.py:414-434)."""
        self.prepare_data(jobids)
        self.gradout = 1 if withgrad else 0
        self.N = np.array(params[self.params[0]].shape, dtype=int)
        self.write_csts(workdir)
        self.write_model(params, workdir)

    def set_backward(self, residuals=None, workdir=None):
        """Provide the adjoint sources for a gradient-only run (SeisCL.py:436-457)."""
        if residuals is not None:
            rec = {}
            for n, word in enumerate(self.to_load_names):
                rec[word + "res"] = np.asarray(residuals[n], dtype=np.float32)
            self._put(self.file_res, rec, workdir)
            self.inputres = 1
        else:
            self.inputres = 0
        self.gradout = 1
        self.write_csts(workdir)

    def callcmd(self, workdir=None):
        """The reference's launch command has no counterpart: the engine is
        called in-process. Returns a one-line description of the call."""
        return "%s: in-process CUDA engine, file %s" % (self.progname, self.file)

    def write_csts(self, workdir=None, filename=None):
        """The constants of ``CSTS`` (SeisCL.py:703-721)."""
        if filename is None:
            filename = self.file_csts
        self._put(filename, {k: self.__dict__[k] for k in CSTS if self.__dict__.get(k) is not None}, workdir)

    def read_csts(self, workdir=None, filename=None):
        """Replace the constants with those of the constants file
        (SeisCL.py:682-701)."""
        if filename is None:
            filename = self.file_csts
        rec = self._get(filename, workdir)
        if rec is None:
            raise SeisCLError('could not read parameter file \n')
        for k, v in rec.items():
            if k in CSTS:
                v = np.asarray(v)
                self.__dict__[k] = v.item() if v.ndim == 0 else v

    def write_model(self, params, workdir=None):
        """Store the model (SeisCL.py:747-763): every name of ``params`` is
        required, arrays are N-shaped ([NZ, NX] or [NZ, NY, NX])."""
        for param in self.params:
            if param not in params:
                raise SeisCLError('Parameter with %s not defined\n' % param)
        self._model = {k: np.asarray(v, dtype=np.float32).copy() for k, v in params.items()}
        self._put(self.file_model, self._model, workdir)

    def write_data(self, data, workdir=None, filename=None):
        """Store observed data (SeisCL.py:658-680); arrays are NT x ntraces."""
        if filename is None:
            filename = self.file_din
        data = dict(data)
        if 'src_pos' not in data:
            data['src_pos'] = self.src_pos
        if 'rec_pos' not in data:
            data['rec_pos'] = self.rec_pos
        if 'src' not in data:
            data['src'] = self.src
        self._put(filename, {k: (None if v is None else np.array(v, copy=True)) for k, v in data.items()}, workdir)

    def prepare_data(self, srcids):
        """Select sources and receivers of ``srcids`` (SeisCL.py:765-808)."""
        if np.issubdtype(type(srcids), np.integer):
            srcids = [srcids]
        srcids = [int(s) for s in np.atleast_1d(srcids)]
        srcels = [ii for ii, el in enumerate(self.src_pos_all[3, :].astype(int)) if el in srcids]
        recels = [g for g, s in enumerate(self.rec_pos_all[3, :].astype(int)) if s in srcids]
        if len(srcels) <= 0:
            raise ValueError('No shot found')
        self.src_pos = self.src_pos_all[:, srcels]
        if self.src_all is None:
            self.src_all = np.stack([self.wavelet_generator()] * self.src_pos_all.shape[1], 1)
        self.src = self.src_all[:, srcels]
        self.rec_pos = self.rec_pos_all[:, recels]
        if self.filter_offset:
            validrec = []
            for ii in range(0, self.rec_pos.shape[1]):
                srcid = np.where(self.src_pos[3, :] == self.rec_pos[3, ii])
                offset = np.sqrt((self.rec_pos[0, ii] - self.src_pos[0, srcid]) ** 2
                                 + (self.rec_pos[1, ii] - self.src_pos[1, srcid]) ** 2
                                 + (self.rec_pos[2, ii] - self.src_pos[2, srcid]) ** 2)
                if self.offmax >= offset >= self.offmin:
                    validrec.append(ii)
            self.rec_pos = self.rec_pos[:, validrec]
            recels = [recels[el] for el in validrec]
        self.rec_pos = np.array(self.rec_pos, dtype=float, copy=True)
        self.rec_pos[4, :] = [x + 1 for x in recels]

    def ricker_wavelet(self, f0=None, NT=None, dt=None, tmin=None):
        """Ricker wavelet of SeisCL.py:810-834."""
        if NT is None:
            NT = self.NT
        if f0 is None:
            f0 = self.f0
        if dt is None:
            dt = self.dt
        if tmin is None:
            tmin = -1.5 / f0
        t = np.linspace(tmin, (NT - 1) * dt + tmin, num=int(NT))
        return ((1.0 - 2.0 * (np.pi ** 2) * (f0 ** 2) * (t ** 2))
                * np.exp(-(np.pi ** 2) * (f0 ** 2) * (t ** 2)))

    def invert_source(self, src, datao, datam, srcid=None):
        """Frequency-domain source estimate of SeisCL.py:725-745."""
        dm = np.fft.fft(datam, axis=0)
        do = np.fft.fft(datao, axis=0)
        s = np.fft.fft(np.squeeze(src), axis=0)
        a = np.sum(np.conj(dm) * do, axis=1) / np.sum(dm * np.conj(dm), axis=1)
        src_new = np.real(np.fft.ifft(a * s[:]))
        if srcid is not None:
            self.src_all[:, srcid] = src_new
        return src_new

    def surface_acquisition_2d(self, dg=2, ds=5, dsx=2, dsz=2, dgsz=0, src_type=100):
        """Regular surface acquisition (SeisCL.py:862-909).

        One shot every ``ds`` cells from ``nab + dsx`` to ``nx - nab - dsx``,
        at ``dsz`` cells below the free surface (or below the absorbing
        layer without one); receivers every ``dg`` cells starting ``dsx``
        cells after the first source, ``dgsz`` cells below the sources.
        Replaces ``src_pos_all``/``rec_pos_all`` and clears ``src_all``."""
        self.src_pos_all = np.empty((5, 0))
        self.rec_pos_all = np.empty((8, 0))
        self.src_all = None
        nx = self.N[1]
        dlx = self.nab + dsx
        dlz = self.nab + dsz if self.freesurf == 0 else dsz
        gx = np.arange(dlx + dsx, nx - dlx, dg) * self.dh
        gz = np.zeros_like(gx) + (dlz + dgsz) * self.dh
        for ii in range(dlx, nx - dlx, ds):
            self._append_shot(ii * self.dh, dlz * self.dh, src_type, gx, gz, 0)

    def crosshole_acquisition_2d(self, dg=2, ds=5, dsx=2, dsz=2):
        """Multi-offset cross-hole acquisition (SeisCL.py:911-952).

        Explosive shots down the left well (``nab + dsx`` cells from the
        left edge) every ``ds`` cells, receivers down the right well every
        ``dg`` cells, both from ``dsz`` cells below the free surface (or the
        absorbing layer). Shots are appended to ``src_pos_all``; receivers
        are flagged with type 2 in row 5 of ``rec_pos_all``."""
        nz, nx = self.N
        dlx = self.nab + dsx
        dlz = self.nab + dsz if self.freesurf == 0 else dsz
        gz = np.arange(dlz, nz - dlz, dg) * self.dh
        gx = np.zeros_like(gz) + (nx - dlx) * self.dh
        for ii in range(dlz, nz - dlz, ds):
            self._append_shot(dlx * self.dh, ii * self.dh, 100, gx, gz, 2)

    def _append_shot(self, xs, zs, src_type, gx, gz, rec_flag):
        idsrc = self.src_pos_all.shape[1]
        self.src_pos_all = np.append(self.src_pos_all, np.array([[xs], [0], [zs], [idsrc], [src_type]], float), axis=1)
        gid = np.arange(len(gx)) + self.rec_pos_all.shape[1] + 1
        zero = np.zeros_like(gx)
        recs = np.stack([gx, zero, gz, zero + idsrc, gid, zero + rec_flag, zero, zero], 0)
        self.rec_pos_all = np.append(self.rec_pos_all, recs, axis=1)

    # ------------------------------------------------------------- reading
    def read_data(self, workdir=None, filename=None, residuals=False):
        """Seismograms (or residuals) of the last run, NT x ntraces each, in
        the order of ``to_load_names`` (SeisCL.py:507-541)."""
        if filename is None:
            filename = self.file_dout
        suf = "res" if residuals else "out"
        mat = self._get(filename, workdir)
        if mat is None:
            raise SeisCLError('Could not read data')
        output = [mat[w + suf] for w in self.to_load_names if w + suf in mat]
        if not output:
            raise SeisCLError('Could not read data: variables not found')
        return output

    def read_movie(self, workdir=None, filename=None):
        """Movie of the last run (SeisCL.py:543-571): for each recorded
        variable that is a wave field, the snapshots taken every ``movout``
        steps, shaped as the reference returns them (N reversed, then
        snapshot, then shot)."""
        if filename is None:
            filename = self.file_movout
        mat = self._get(filename, workdir)
        if mat is None:
            raise SeisCLError('Could not read data')
        output = [np.transpose(mat["mov" + w]) for w in self.to_load_names if "mov" + w in mat]
        if not output:
            raise SeisCLError('Could not read data: variables not found')
        return output

    def read_grad(self, workdir=None, param_names=None, filename=None):
        """Gradients of the last run, N-shaped, zeroed in the absorbing
        layers when ``cropgrad`` (SeisCL.py:573-602)."""
        if filename is None:
            filename = self.file_gout
        if param_names is None:
            param_names = self.params
        mat = self._get(filename, workdir)
        if mat is None:
            raise SeisCLError('Could not read grad')
        try:
            output = [np.array(mat['grad' + name], copy=True) for name in param_names]
        except KeyError as exc:
            raise SeisCLError('Could not read grad: %s' % exc) from exc
        if self.cropgrad:
            for o in output:
                if self.freesurf == 0:
                    o[:self.nab, ...] = 0
                o[-self.nab:, ...] = 0
                o[:, :self.nab, ...] = 0
                o[:, -self.nab:, ...] = 0
        return output

    def read_Hessian(self, workdir=None, param_names=None, filename=None):
        """Approximate Hessian of the last run (``Hout=1``), as read_grad
        (SeisCL.py:604-634)."""
        if filename is None:
            filename = self.file_gout
        if param_names is None:
            param_names = self.params
        mat = self._get(filename, workdir)
        if mat is None:
            raise SeisCLError('Could not read Hessian')
        try:
            output = [np.array(mat['H' + name], copy=True) for name in param_names]
        except KeyError as exc:
            raise SeisCLError('Could not read Hessian') from exc
        if self.cropgrad:
            for o in output:
                if self.freesurf == 0:
                    o[:self.nab, ...] = 0
                o[-self.nab:, ...] = 0
                o[:, :self.nab, ...] = 0
                o[:, -self.nab:, ...] = 0
        return output

    def read_rms(self, workdir=None, filename=None):
        """(rms / rms_norm, rms_norm) of the last run (SeisCL.py:636-656)."""
        if filename is None:
            filename = self.file_rms
        mat = self._get(filename, workdir)
        if mat is None:
            raise SeisCLError('Forward modeling failed, could not read rms\n')
        return mat['rms'][0] / mat['rms_norm'][0], mat['rms_norm'][0]

    # ----------------------------------------------------------- execution
    def _engine_config(self) -> engine.Config:
        N = [int(v) for v in np.atleast_1d(self.N)]
        bpt = int(self.back_prop_type)
        if bpt not in (1, 2):
            raise SeisCLError("Error: back_prop_type must be 1 (backpropagation) or 2 (DFT)")
        freqs = tuple(float(v) for v in np.atleast_1d(self.gradfreqs).ravel())
        if bpt == 2 and self.gradout and not freqs:
            # read_hdf5.c:546-549 requires /gradfreqs for the DFT gradient
            raise SeisCLError("Error: back_prop_type=2 needs gradfreqs")
        for flag in ("gradsrcout",):
            if getattr(self, flag):
                raise SeisCLError("Error: %s is not provided by this engine" % flag)
        return engine.Config(
            N=N, ND=int(self.ND), dh=float(self.dh), dt=float(self.dt), NT=int(self.NT), L=int(self.L),
            f0=float(self.f0), FL=tuple(np.atleast_1d(self.FL).astype(float)), FDORDER=int(self.FDORDER),
            MAXRELERROR=int(self.MAXRELERROR), freesurf=int(self.freesurf), abs_type=int(self.abs_type),
            VPPML=float(self.VPPML), NPOWER=float(self.NPOWER), FPML=float(self.FPML),
            K_MAX_CPML=float(self.K_MAX_CPML), nab=int(self.nab), abpc=float(self.abpc),
            tmin=self._steps(self.tmin), tmax=self._steps(self.tmax),
            param_type=int(self.param_type), restype=int(self.restype),
            precision="fp16" if int(self.FP16) >= 2 else "fp32",
            field_precision="fp16" if (int(self.FP16) >= 2 and int(self.ND) in (2, 3) and int(self.L) <= 3
                                       and not self.gradout) else "fp32",
            back_prop_type=bpt, gradfreqs=freqs if bpt == 2 else (),
            hout=1 if (self.Hout and self.gradout) else 0)

    def _steps(self, seconds) -> int:
        """A time in seconds as a step count, FP32 quotient truncated
        (read_hdf5.c:524-529); 0 keeps the default."""
        f = np.float32(seconds)
        return int(f / np.float32(self.dt)) if f > 0 else 0

    def _get_plan(self) -> engine.Plan:
        cfg = self._engine_config()
        key = repr(cfg)
        if self._plan is None or self._plan_key != key:
            if self._plan is not None:
                self._plan.close()
            try:
                self._plan = engine.Plan(cfg)
            except engine.SeisCLEngineError as exc:
                raise SeisCLError(str(exc)) from exc
            self._plan_key = key
        return self._plan

    def _host_model(self):
        """Model arrays in engine layout (x slowest, z fastest)."""
        m = self._model
        if m is None:
            raise SeisCLError("Error: Could not open the input file model")
        names = {0: ("vp", "vs"), 1: ("M", "mu"), 2: ("Ip", "Is")}[self.param_type]
        get = lambda k: None if k not in m else np.ascontiguousarray(np.transpose(m[k]), dtype=np.float32)
        for k in self.params:
            if tuple(np.shape(m[k])) != tuple(int(v) for v in np.atleast_1d(self.N)):
                raise SeisCLError("Error: Variable %s must have dimensions in N\n" % k)
        return get(names[0]), get(names[1]), get("rho"), get("taup"), get("taus")

    def _shots(self):
        """Split the selected sources and receivers into shots by srcid,
        ascending as read_hdf5.c:357-393 requires."""
        sp = np.asarray(self.src_pos, dtype=float)
        rp = np.asarray(self.rec_pos, dtype=float)
        ids = sp[3].astype(int)
        if np.any(np.diff(ids) < 0):
            raise SeisCLError("Sources ids must be sorted in ascending order")
        if rp.shape[1] and np.any(np.diff(rp[3].astype(int)) < 0):
            raise SeisCLError("Src ids in rec_pos must be sorted in ascending order")
        shots = []
        for sid in np.unique(ids):
            si = np.nonzero(ids == sid)[0]
            gi = np.nonzero(rp[3].astype(int) == sid)[0]
            shots.append((sid, si, gi))
        if len(np.unique(rp[3].astype(int))) != len(shots):
            raise SeisCLError("Error: Number of sources ids in src_pos and rec_pos are not the same")
        return shots

    def _outputs(self, din, resin):
        """Variables to record: from the residual file for a gradient-only
        run, from the observed data when a misfit is needed, else from
        ``seisout`` (read_hdf5.c:640-766, assign_modeling_case.c:1242-1322)."""
        allowed = _VARS[int(self.ND)]
        if self.inputres and self.gradout:
            if resin is None:
                raise SeisCLError("Error: Could not open the residuals file")
            outs = [v for v in allowed if v + "res" in resin]
            if not outs:
                raise SeisCLError("Error: Cannot output without the residuals")
            return outs
        if not self.inputres and (self.rmsout or self.resout or self.gradout):
            if din is None:
                raise SeisCLError("Error: Could not open the input file for data_in")
            outs = [v for v in allowed if v in din]
            if not outs:
                raise SeisCLError("Error: Cannot output gradient, rms or residuals without reference data")
            return outs
        if self.seisout == 2 and int(self.ND) == 21:
            raise SeisCLError("Error: Cannot output pressure for SH modeling")
        names = self.to_load_names or []
        return [v for v in names if v in allowed]

    def _residuals(self, out, obs, rp_shot, NT, tmax):
        """Adjoint sources and misfit of one shot, src/residuals.c:58-450
        (restype 0) and residuals.c:26-56 (restype 1). ``out``/``obs`` map a
        name to [nrec][NT] arrays. Returns (res, rms, rmsnorm)."""
        names = list(out)
        out = {k: np.array(v, dtype=np.float32, copy=True) for k, v in out.items()}
        obs = {k: np.array(v, dtype=np.float32, copy=True) for k, v in obs.items()}
        if self.restype == 1:
            res = {k: np.zeros_like(out[k]) for k in names}
            for k in names:
                res[k][:, :tmax] = obs[k][:, :tmax]
            return res, 0.0, 0.0
        if self.restype != 0:
            raise SeisCLError("Error: Unknown restype")
        if self.fmax > 0 or self.fmin > 0:
            for k in names:
                out[k] = butterworth(out[k], self.fmin, self.fmax, self.dt, tmax)
                obs[k] = butterworth(obs[k], self.fmin, self.fmax, self.dt, tmax)
        tmin = self._steps(self.tmin)
        nrec = out[names[0]].shape[0]
        sc = np.ones(nrec, np.float64)
        sc0 = np.ones(nrec, np.float64)
        if self.scalerms or self.scaleshot or self.scalermsnorm:
            e = sum((out[k][:, tmin:tmax].astype(np.float64) ** 2).sum(1) for k in names)
            e0 = sum((obs[k][:, tmin:tmax].astype(np.float64) ** 2).sum(1) for k in names)
            sc = np.sqrt(1.0 / e)
            sc0 = np.sqrt(1.0 / e0)
            ws = 0.0
            if self.scaleshot:
                ws = 1.0 / np.sqrt(np.sum(1.0 / sc0 ** 2))
                sc[:] = ws
                sc0[:] = ws
            if self.scalerms:
                ws = 1.0 / np.sqrt(np.sum(1.0 / sc0 ** 2))
                sc = sc * ws / sc0
                sc0[:] = ws
            for k in names:
                out[k][:, tmin:tmax] *= sc[:, None].astype(np.float32)
                obs[k][:, tmin:tmax] *= sc0[:, None].astype(np.float32)
        rmsnorm_sc = None
        if self.scalerms or self.scalermsnorm:
            acc = sum((out[k][:, tmin:tmax].astype(np.float64)
                       * (out[k][:, tmin:tmax] - obs[k][:, tmin:tmax])).sum(1) for k in names)
            if self.scalerms:
                acc = acc * (ws / sc0 / ws) ** 2
            rmsnorm_sc = 1.0 - acc
        rms = 0.0
        rmsnorm = 0.0
        res = {}
        dft = int(self.back_prop_type) == 2
        if dft:
            # misfit at the gradient frequencies only (residuals.c:254-410):
            # |FFT|^2 of the residual and of the data at bin int(f*nfft*dt + 1)
            nfft = next_fast_size(tmax)
            bins = [int(np.float32(f) * nfft * np.float32(self.dt) + 1)
                    for f in np.atleast_1d(self.gradfreqs).ravel()]
        for k in names:
            o = out[k][:, :tmax].astype(np.float64)
            d = obs[k][:, :tmax].astype(np.float64)
            if dft:
                R = np.fft.rfft(d - o, n=nfft, axis=1)[:, bins]
                D = np.fft.rfft(d, n=nfft, axis=1)[:, bins]
                rms += float((np.abs(R) ** 2).sum())
                rmsnorm += float((np.abs(D) ** 2).sum())
            else:
                rms += float(((d - o) ** 2).sum())
                rmsnorm += float((d ** 2).sum())
            if not np.isfinite(rms):
                # src/residuals.c:444-448
                raise SeisCLError("Simulation has become unstable, stopping\n")
            r = np.zeros_like(out[k])
            if rmsnorm_sc is not None:
                r[:, :tmax] = sc[:, None] * ((1.0 - rmsnorm_sc)[:, None] * o - d)
            else:
                r[:, :tmax] = sc[:, None] * (o - d)
            res[k] = r
        return res, rms, rmsnorm

    def execute(self, workdir=None):
        """Run the job prepared by ``set_forward``/``set_backward`` on the
        current CUDA device and store its outputs (SeisCL.py:487-505,
        src/time_stepping.c:693-900). Returns a short log."""
        t0 = time.perf_counter()
        if self.use_files:
            model = self._get(self.file_model, workdir)
            if model is None:
                raise SeisCLError("Error: Could not open the input file model")
            self._model = model
        plan = self._get_plan()
        nd = int(self.ND)
        NT = int(self.NT)
        try:
            plan.set_model(*self._host_model())
        except engine.SeisCLEngineError as exc:
            raise SeisCLError(str(exc)) from exc
        tmax = plan.tmax
        din = self._get(self.file_din, workdir)
        resin = self._get(self.file_res, workdir) if self.inputres else None
        if self.inputres and self.resout:
            raise SeisCLError("Error: Cannot input and output residuals simultaneously")
        outs = self._outputs(din, resin)
        shots = self._shots()
        # shots of this rank when running one process per GPU (time_stepping.c:705-722)
        rank, world, _ = shots_mod.dist_context()
        smin, smax = shots_mod.shot_range(len(shots), rank, world)
        sp_all = np.asarray(self.src_pos, dtype=np.float32).T
        src_all = np.asarray(self.src, dtype=np.float32).T
        rp_all = np.asarray(self.rec_pos, dtype=np.float32).T
        ntr = rp_all.shape[0]
        seis = {k: np.zeros((ntr, NT), np.float32) for k in outs}
        resid = {k: np.zeros((ntr, NT), np.float32) for k in outs}
        need_res = not self.inputres and (self.gradout or self.rmsout or self.resout)
        rms = rmsnorm = 0.0
        if self.gradout:
            plan.zero_gradient()
        movout = int(self.movout)
        movies = None
        if movout > 0:
            # [shot][snapshot][nx][(ny)][nz] per filmed variable (writehdf5.c:295-310)
            films = [k for k in outs if k != "p" or nd == 22]
            shape = (len(shots), NT // movout) + tuple(int(v) for v in np.atleast_1d(self.N)[::-1])
            movies = {k: np.zeros(shape, np.float32) for k in films}
        pending = None   # (shot index, arrays the last shot's runs filled)

        def keep_movie():
            if pending is not None:
                for k, v in pending[1].items():
                    movies[k][pending[0]] = v
        try:
            for ishot, (sid, si, gi) in enumerate(shots):
                if not smin <= ishot < smax:
                    continue
                keep_movie()
                sp, src, rp = sp_all[si], src_all[si], rp_all[gi]
                if movies is not None:
                    pending = (ishot, plan.set_movie(movout, list(movies)))
                if self.inputres and self.gradout:
                    res = {k: np.ascontiguousarray(np.transpose(resin[k + "res"]), dtype=np.float32)[
                        rp[:, 4].astype(int) - 1] for k in outs}
                    plan.forward(sp, src, rp, [], save_boundaries=True)
                else:
                    d = plan.forward(sp, src, rp, outs, save_boundaries=bool(self.gradout))
                    for k in outs:
                        seis[k][gi] = d[k]
                    if not need_res:
                        continue
                    obs = {k: np.ascontiguousarray(np.transpose(din[k]), dtype=np.float32)[rp[:, 4].astype(int) - 1]
                           for k in outs}
                    res, r1, r2 = self._residuals(d, obs, rp, NT, tmax)
                    rms += r1
                    rmsnorm += r2
                    for k in outs:
                        resid[k][gi] = res[k]
                    if not self.gradout:
                        continue
                res = plan.residual_scale(rp, res)
                plan.adjoint(sp, src, rp, res)
            keep_movie()
        except engine.SeisCLEngineError as exc:
            raise SeisCLError(str(exc)) from exc
        finally:
            if movies is not None:
                plan.set_movie(0)
        if world > 1:
            # every rank filled only the traces of its own shots, a contiguous
            # block of rows (shots and traces ascend by srcid): gather the
            # blocks (Out_MPI.c:70-160); the misfit is summed, and the
            # gradient below too, after the chain rule, which is linear in the
            # accumulated kernels
            rows = [gi for _, _, gi in shots[smin:smax]]
            lo = int(min((r.min() for r in rows if len(r)), default=0))
            hi = int(max((r.max() + 1 for r in rows if len(r)), default=lo))
            tr = {"seis_" + k: v for k, v in seis.items()}
            tr.update({"res_" + k: v for k, v in resid.items()})
            tr = shots_mod.gather_rows(tr, lo, hi)
            seis = {k: tr["seis_" + k] for k in seis}
            resid = {k: tr["res_" + k] for k in resid}
            if movies is not None:
                movies = shots_mod.gather_rows(movies, smin, smax)
            rms, rmsnorm = (float(v) for v in shots_mod.allreduce_sum({"rms": np.array([rms, rmsnorm])})["rms"])
        if not (self.inputres and self.gradout):
            dout = {k + "out": np.ascontiguousarray(seis[k].T) for k in outs}
            if self.resout and not self.inputres:
                dout.update({k + "res": np.ascontiguousarray(resid[k].T) for k in outs})
            dout["src_pos"] = np.asarray(self.src_pos).copy()
            dout["rec_pos"] = np.asarray(self.rec_pos).copy()
            if self.seisout or self.resout:
                self._put(self.file_dout, dout, workdir)
        if movies is not None:
            self._put(self.file_movout, {"mov" + k: v for k, v in movies.items()}, workdir)
        if self.rmsout:
            # 1 x 1 datasets (writehdf5.c:249-257)
            self._put(self.file_rms, {"rms": np.array([[np.sqrt(rms)]], np.float32),
                                      "rms_norm": np.array([[np.sqrt(rmsnorm)]], np.float32)}, workdir)
        if self.gradout:
            g = plan.gradient(transform=True)
            H = plan.hessian(transform=True) if self.Hout else None
            if world > 1:
                g = shots_mod.allreduce_sum(g)
                if H is not None:
                    H = shots_mod.allreduce_sum(H)
            shape = tuple(int(v) for v in np.atleast_1d(self.N))
            names = {0: ("vp", "vs"), 1: ("M", "mu"), 2: ("Ip", "Is")}[self.param_type]
            gout = {}
            qnames = ("taup", "taus") if int(self.L) > 0 else ()
            for name in (names[0], names[1], "rho") + qnames:
                if nd == 22 and name in (names[1], "taus"):
                    continue
                if nd == 21 and name == names[0]:
                    continue
                # the boundary-saving gradient leaves taup/taus at zero (writehdf5.c:262-275)
                v = g[name] if name in g else np.zeros_like(g["rho"])
                gout["grad" + name] = np.ascontiguousarray(np.transpose(v)).reshape(shape)
                if H is not None:
                    v = H[name] if name in H else np.zeros_like(H["rho"])
                    gout["H" + name] = np.ascontiguousarray(np.transpose(v)).reshape(shape)
            self._put(self.file_gout, gout, workdir)
        ms = (time.perf_counter() - t0) * 1e3
        return "%d shot(s) (%d on rank %d of %d), %d trace(s), %d time steps: %.1f ms\n" % (
            len(shots), smax - smin, rank, world, ntr, NT, ms)

    def close(self):
        if self._plan is not None:
            self._plan.close()
            self._plan = None
