"""Dense spin-orbital reference implementations (test helper): MP2 and CCSD
with the Stanton-Gauss intermediates (J. Chem. Phys. 94, 4334 (1991)) on full
antisymmetrised integral tensors.  Small systems only."""
import numpy as np


def spin_orbital(space, f, eri_elems):
    """Fock and <pq||rs> over spin orbitals ordered as the engine's type-local
    indices: holes 2*i+s (i in hole order), then particles 2*a+s."""
    orbs = np.concatenate([space.hole, space.part])
    n = 2 * len(orbs)
    sp = np.arange(n) % 2
    p = orbs[np.arange(n) // 2]
    F = f[p[:, None], p[None, :]] * (sp[:, None] == sp[None, :])
    P, Q, R, S = np.meshgrid(p, p, p, p, indexing="ij")
    s1, s2, s3, s4 = np.meshgrid(sp, sp, sp, sp, indexing="ij")
    direct = eri_elems(P, R, Q, S) * ((s1 == s3) & (s2 == s4))
    exch = eri_elems(P, S, Q, R) * ((s1 == s4) & (s2 == s3))
    return F, direct - exch, 2 * len(space.hole)


def ccsd(F, W, no, maxiter=50, conv=1e-10, mp2_only=False, callback=None):
    o, v = slice(0, no), slice(no, F.shape[0])
    fo, fv = np.diag(F)[o], np.diag(F)[v]
    Dia = fo[:, None] - fv[None, :]
    Dijab = fo[:, None, None, None] + fo[None, :, None, None] - fv[None, None, :, None] - \
        fv[None, None, None, :]
    nv = F.shape[0] - no
    t1 = np.zeros((no, nv))
    t2 = np.zeros((no, no, nv, nv))
    fov = F[o, v]
    Woooo, Wooov, Woovv = W[o, o, o, o], W[o, o, o, v], W[o, o, v, v]
    Wovov, Wovvv, Wvvvv = W[o, v, o, v], W[o, v, v, v], W[v, v, v, v]
    Wvvov, Wovoo = W[v, v, o, v], W[o, v, o, o]
    Wvvoo = W[v, v, o, o]
    Woovo = W[o, o, v, o]
    Wovvo = W[o, v, v, o]
    hist = []
    E = 0.0
    for it in range(1, maxiter + 1):
        tau = t2 + np.einsum("ia,jb->ijab", t1, t1) - np.einsum("ib,ja->ijab", t1, t1)
        taut = t2 + 0.5 * (np.einsum("ia,jb->ijab", t1, t1) - np.einsum("ib,ja->ijab", t1, t1))
        E = np.einsum("ia,ia", fov, t1) + 0.25 * np.einsum("ijab,ijab", Woovv, tau)
        if mp2_only:
            r2 = Wvvoo.transpose(2, 3, 0, 1) + np.einsum("be,ijae->ijab", F[v, v], t2) - \
                np.einsum("ae,ijbe->ijab", F[v, v], t2) - np.einsum("mj,imab->ijab", F[o, o], t2) \
                + np.einsum("mi,jmab->ijab", F[o, o], t2)
            E = 0.25 * np.einsum("ijab,ijab", Woovv, t2)
            rn = np.linalg.norm(r2) / 2.0  # unique elements only: each appears 4 times
            hist.append((it, E, rn))
            if callback:
                callback(it, E, rn)
            if rn < conv:
                break
            t2 = t2 + r2 / Dijab
            continue
        Fae = F[v, v] - 0.5 * np.einsum("me,ma->ae", fov, t1) + \
            np.einsum("mf,mafe->ae", t1, Wovvv) - 0.5 * np.einsum("mnaf,mnef->ae", taut, Woovv)
        Fmi = F[o, o] + 0.5 * np.einsum("ie,me->mi", t1, fov) + \
            np.einsum("ne,mnie->mi", t1, Wooov) + 0.5 * np.einsum("inef,mnef->mi", taut, Woovv)
        Fme = fov + np.einsum("nf,mnef->me", t1, Woovv)
        Wmnij = Woooo + np.einsum("je,mnie->mnij", t1, Wooov) - \
            np.einsum("ie,mnje->mnij", t1, Wooov) + 0.25 * np.einsum("ijef,mnef->mnij", tau, Woovv)
        Wabef = Wvvvv - np.einsum("mb,amef->abef", t1, W[v, o, v, v]) + \
            np.einsum("ma,bmef->abef", t1, W[v, o, v, v]) + \
            0.25 * np.einsum("mnab,mnef->abef", tau, Woovv)
        Wmbej = Wovvo + np.einsum("jf,mbef->mbej", t1, Wovvv) - \
            np.einsum("nb,mnej->mbej", t1, Woovo) - \
            np.einsum("jnfb,mnef->mbej", 0.5 * t2 + np.einsum("jf,nb->jnfb", t1, t1), Woovv)
        r1 = fov + np.einsum("ie,ae->ia", t1, Fae) - np.einsum("ma,mi->ia", t1, Fmi) + \
            np.einsum("imae,me->ia", t2, Fme) - np.einsum("nf,naif->ia", t1, Wovov) - \
            0.5 * np.einsum("imef,maef->ia", t2, Wovvv) - \
            0.5 * np.einsum("mnae,nmei->ia", t2, W[o, o, v, o])
        Fbe = Fae - 0.5 * np.einsum("mb,me->be", t1, Fme)
        Fmj = Fmi + 0.5 * np.einsum("je,me->mj", t1, Fme)
        x = np.einsum("ijae,be->ijab", t2, Fbe)
        r2 = Woovv.transpose(0, 1, 2, 3).copy() * 0 + W[o, o, v, v]
        r2 = r2 + x - x.transpose(0, 1, 3, 2)
        x = np.einsum("imab,mj->ijab", t2, Fmj)
        r2 = r2 - x + x.transpose(1, 0, 2, 3)
        r2 = r2 + 0.5 * np.einsum("mnab,mnij->ijab", tau, Wmnij) + \
            0.5 * np.einsum("ijef,abef->ijab", tau, Wabef)
        x = np.einsum("imae,mbej->ijab", t2, Wmbej) - \
            np.einsum("ie,ma,mbej->ijab", t1, t1, Wovvo)
        r2 = r2 + x - x.transpose(0, 1, 3, 2) - x.transpose(1, 0, 2, 3) + x.transpose(1, 0, 3, 2)
        x = np.einsum("ie,abej->ijab", t1, W[v, v, v, o])
        r2 = r2 + x - x.transpose(1, 0, 2, 3)
        x = np.einsum("ma,mbij->ijab", t1, Wovoo)
        r2 = r2 - x + x.transpose(0, 1, 3, 2)
        # full residuals (diagonal Fock included through Fae, Fmi)
        rn = np.sqrt(np.sum(r1 ** 2) + np.sum(r2 ** 2) / 4.0)
        hist.append((it, E, rn))
        if callback:
            callback(it, E, rn)
        if rn < conv:
            break
        t1 = t1 + r1 / Dia
        t2 = t2 + r2 / Dijab
    return E, hist
