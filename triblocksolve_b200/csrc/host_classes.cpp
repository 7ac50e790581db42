/*
 * host_classes.cpp -- Platform / Mesh / Jacobian host classes over the C ABI.
 */
#include "Jacobian.hxx"
#include "Mesh.hxx"

#include <algorithm>
#include <cstring>

/* ------------------------------------------------------------- Platform */

Platform::Platform(int mode, int dev) : compute_mode(mode), device_id(dev) {
    if (mode != TBS_CUDA_MODE)
        throw std::runtime_error("compute_mode " + std::to_string(mode) +
                                 " is not available: this build runs only on CUDA (mode 2)");
    int st = tbs_create(dev, &ctx);
    if (st != TBS_OK) throw std::runtime_error(tbs_last_error(nullptr));
}

Platform::~Platform() {
    if (ctx) tbs_destroy(ctx);
}

size_t Platform::memoryAllocated() const {
    size_t b = 0;
    if (ctx) tbs_memory_allocated(ctx, &b);
    return b;
}

/* ----------------------------------------------------------------- Mesh */

void Mesh::finish_sizes() {
    /* src/Mesh.cxx:45-59 and :67-68 */
    nbytes = epoint.size() + ef.size() + fc.size() + linesize.size() + linepoint.size() +
             lines.size() + lineface.size();
    max_line_nelem = 0;
    for (int v : linesize) max_line_nelem = std::max(max_line_nelem, v);
}

bool Mesh::fromFile(const char *path) {
    int hdr[6];
    if (tbs_read_mesh_header(path, hdr) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    nvar = hdr[0];
    nelem = hdr[1];
    nintface = hdr[2];
    eftot = hdr[3];
    nline = hdr[4];
    nlineelem = hdr[5];
    ef.resize(eftot);
    fc.resize(2 * (size_t)nintface);
    epoint.resize((size_t)nelem + 1);
    lines.resize(nlineelem);
    linesize.resize(nline);
    linepoint.resize((size_t)nline + 1);
    lineface.resize(nlineelem);
    if (tbs_read_mesh(path, hdr, epoint.data(), ef.data(), fc.data(), linesize.data(),
                      linepoint.data(), lines.data(), lineface.data()) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    finish_sizes();
    return true;
}

bool Mesh::fromStructured(int L, int K, int nv) {
    int hdr[6];
    if (tbs_gen_structured_header(L, K, nv, hdr) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    nvar = hdr[0];
    nelem = hdr[1];
    nintface = hdr[2];
    eftot = hdr[3];
    nline = hdr[4];
    nlineelem = hdr[5];
    ef.resize(eftot);
    fc.resize(2 * (size_t)nintface);
    epoint.resize((size_t)nelem + 1);
    lines.resize(nlineelem);
    linesize.resize(nline);
    linepoint.resize((size_t)nline + 1);
    lineface.resize(nlineelem);
    if (tbs_gen_structured_mesh(L, K, epoint.data(), ef.data(), fc.data(), linesize.data(),
                                linepoint.data(), lines.data(), lineface.data()) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    finish_sizes();
    return true;
}

bool Mesh::toFile(const char *path) const {
    int hdr[6] = {nvar, nelem, nintface, eftot, nline, nlineelem};
    return tbs_write_mesh(path, hdr, epoint.data(), ef.data(), fc.data(), linesize.data(),
                          linepoint.data(), lines.data(), lineface.data()) == TBS_OK;
}

void Mesh::setupDevice(Platform &gpu) { gpu_ = &gpu; }

void Mesh::toDevice() {
    if (!gpu_) throw std::runtime_error("Mesh::toDevice before setupDevice");
    int st = tbs_set_mesh(gpu_->ctx, nvar, nelem, nintface, eftot, nline, nlineelem, epoint.data(),
                          ef.data(), fc.data(), linesize.data(), linepoint.data(), lines.data(),
                          lineface.data());
    if (st != TBS_OK) throw std::runtime_error(tbs_last_error(gpu_->ctx));
}

void Mesh::fromDevice() { /* the mesh is never modified on the device */ }

/* ------------------------------------------------------------- Jacobian */

void Jacobian::size_arrays(int nlineelem) {
    /* src/Jacobian.cxx:36-61 */
    const size_t nb = (size_t)nvar * nvar;
    jacDLU.assign(nb * nelem, 0.0);
    jacD.assign(nb * nelem, 0.0);
    jacO1.assign(nb * nintface, 0.0);
    jacO2.assign(nb * nintface, 0.0);
    rhs.assign((size_t)nvar * nelem, 0.0);
    U0.assign((size_t)nvar * nelem, 0.0);
    U.assign((size_t)nvar * nelem, 0.0);
    dU.assign((size_t)nvar * nelem, 0.0);
    res.assign((size_t)nvar * nelem, 0.0);
    DinvC.assign(nb * nelem, 0.0);
    A.assign(nb * nlineelem, 0.0);
    nbytes = jacD.size() + jacO1.size() + jacO2.size() + rhs.size() + U0.size() + U.size() +
             dU.size() + res.size();
}

bool Jacobian::fromFile(int nlineelem, const char *path) {
    int hdr[3];
    if (tbs_read_jacobian_header(path, hdr) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    nvar = hdr[0];
    nelem = hdr[1];
    nintface = hdr[2];
    size_arrays(nlineelem);
    if (tbs_read_jacobian(path, hdr, jacD.data(), jacO1.data(), jacO2.data(), rhs.data(),
                          U0.data()) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    return true;
}

bool Jacobian::fromGenerator(const Mesh &mesh, double shift, uint64_t seed) {
    nvar = mesh.nvar;
    nelem = mesh.nelem;
    nintface = mesh.nintface;
    size_arrays(mesh.nlineelem);
    if (tbs_gen_jacobian(nvar, nelem, nintface, shift, seed, jacD.data(), jacO1.data(),
                         jacO2.data(), rhs.data(), U0.data()) != TBS_OK) {
        error = tbs_last_error(nullptr);
        return false;
    }
    return true;
}

bool Jacobian::toFile(const char *path) const {
    int hdr[3] = {nvar, nelem, nintface};
    return tbs_write_jacobian(path, hdr, jacD.data(), jacO1.data(), jacO2.data(), rhs.data(),
                              U0.data()) == TBS_OK;
}

void Jacobian::assembleTriBlocks(Mesh &mesh) {
    /* src/Jacobian.cxx:91-116 */
    const size_t bs = (size_t)nvar * nvar;
    if (A.size() < bs * (size_t)mesh.nelem) A.resize(bs * (size_t)mesh.nelem, 0.0);
    for (int l = 0; l < mesh.nline; ++l) {
        for (int k = 1; k < mesh.linesize[l]; ++k) {
            const int m = mesh.linepoint[l] + k;
            const int f = mesh.lineface[m];
            const int e = mesh.lines[m];
            const int e1 = mesh.fc[2 * f];
            const double *src = (e == e1) ? &jacO2[bs * f] : &jacO1[bs * f];
            std::memcpy(&A[bs * e], src, bs * sizeof(double));
        }
    }
}

void Jacobian::resizeBlockSize(int nvar_new) {
    /* src/Jacobian.cxx:153-238; the array rules are in tbs_resize_block_size */
    const int nvar_old = nvar;
    if (nvar_new == nvar) return;
    const size_t bn = (size_t)nvar_new * nvar_new;
    std::vector<double> D(bn * nelem), O1(bn * nintface), O2(bn * nintface);
    std::vector<double> r((size_t)nvar_new * nelem), u0((size_t)nvar_new * nelem);
    if (tbs_resize_block_size(nvar_old, nvar_new, nelem, nintface, jacD.data(), jacO1.data(),
                              jacO2.data(), rhs.data(), U0.data(), D.data(), O1.data(), O2.data(),
                              r.data(), u0.data()) != TBS_OK)
        throw std::runtime_error(tbs_last_error(nullptr));
    nvar = nvar_new;
    jacD.swap(D);
    jacO1.swap(O1);
    jacO2.swap(O2);
    rhs.swap(r);
    U0.swap(u0);
    U.resize((size_t)nvar * nelem);
    jacDLU.resize(bn * nelem);
    dU.resize((size_t)nvar * nelem);
    res.resize((size_t)nvar * nelem);
    A.resize(bn * nelem);
}

void Jacobian::setupDevice(Platform &gpu) { gpu_ = &gpu; }

void Jacobian::toDevice() {
    if (!gpu_) throw std::runtime_error("Jacobian::toDevice before setupDevice");
    int st = tbs_set_jacobian(gpu_->ctx, jacD.data(), jacO1.data(), jacO2.data(), rhs.data(),
                              U0.data());
    if (st != TBS_OK) throw std::runtime_error(tbs_last_error(gpu_->ctx));
}

void Jacobian::fromDevice() {
    if (!gpu_) throw std::runtime_error("Jacobian::fromDevice before setupDevice");
    if (tbs_get_solution(gpu_->ctx, U.data()) != TBS_OK ||
        tbs_get_residual(gpu_->ctx, res.data()) != TBS_OK ||
        tbs_get_update(gpu_->ctx, dU.data()) != TBS_OK)
        throw std::runtime_error(tbs_last_error(gpu_->ctx));
}
