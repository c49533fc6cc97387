// ORACLE-ONLY: the `_galsim` extension module init for the reference build used as a
// checker.  It registers the reference's own pybind11 bindings (pysrc/*.cpp) for every
// part that compiles here.  Left out, because their sources need Eigen or other code that
// is not installed: SBShapelet (Laguerre), RealGalaxy and HSM.  None of them is on the
// FFT drawing path.  The reference's own pysrc/module.cpp is not used because it
// registers those three as well.
#include "Python.h"
#include "PyBind11Helper.h"

namespace galsim {
    void pyExportBounds(py::module&);
    void pyExportPhotonArray(py::module&);
    void pyExportImage(py::module&);
    void pyExportSBProfile(py::module&);
    void pyExportSBAdd(py::module&);
    void pyExportSBConvolve(py::module&);
    void pyExportSBDeconvolve(py::module&);
    void pyExportSBFourierSqrt(py::module&);
    void pyExportSBTransform(py::module&);
    void pyExportSBBox(py::module&);
    void pyExportSBGaussian(py::module&);
    void pyExportSBDeltaFunction(py::module&);
    void pyExportSBExponential(py::module&);
    void pyExportSBSersic(py::module&);
    void pyExportSBSpergel(py::module&);
    void pyExportSBMoffat(py::module&);
    void pyExportSBAiry(py::module&);
    void pyExportSBInterpolatedImage(py::module&);
    void pyExportSBKolmogorov(py::module&);
    void pyExportSBInclinedExponential(py::module&);
    void pyExportSBInclinedSersic(py::module&);
    void pyExportSBVonKarman(py::module&);
    void pyExportSBSecondKick(py::module&);
    void pyExportRandom(py::module&);
    void pyExportTable(py::module&);
    void pyExportInterpolant(py::module&);
    void pyExportCDModel(py::module&);
    void pyExportSilicon(py::module&);
    void pyExportWCS(py::module&);
    void pyExportUtilities(py::module&);
    namespace integ { void pyExportInteg(py::module&); }
    namespace math {
        void pyExportBessel(py::module&);
        void pyExportHorner(py::module&);
    }
}

PYBIND11_MODULE(_galsim, m)
{
    galsim::pyExportBounds(m);
    galsim::pyExportPhotonArray(m);
    galsim::pyExportImage(m);
    galsim::pyExportSBProfile(m);
    galsim::pyExportSBAdd(m);
    galsim::pyExportSBConvolve(m);
    galsim::pyExportSBDeconvolve(m);
    galsim::pyExportSBFourierSqrt(m);
    galsim::pyExportSBTransform(m);
    galsim::pyExportSBBox(m);
    galsim::pyExportSBGaussian(m);
    galsim::pyExportSBDeltaFunction(m);
    galsim::pyExportSBExponential(m);
    galsim::pyExportSBSersic(m);
    galsim::pyExportSBSpergel(m);
    galsim::pyExportSBMoffat(m);
    galsim::pyExportSBAiry(m);
    galsim::pyExportSBInterpolatedImage(m);
    galsim::pyExportSBKolmogorov(m);
    galsim::pyExportSBInclinedExponential(m);
    galsim::pyExportSBInclinedSersic(m);
    galsim::pyExportSBVonKarman(m);
    galsim::pyExportSBSecondKick(m);
    galsim::pyExportRandom(m);
    galsim::pyExportTable(m);
    galsim::pyExportInterpolant(m);
    galsim::pyExportCDModel(m);
    galsim::pyExportSilicon(m);
    galsim::pyExportWCS(m);
    galsim::pyExportUtilities(m);
    galsim::integ::pyExportInteg(m);
    galsim::math::pyExportBessel(m);
    galsim::math::pyExportHorner(m);
}
