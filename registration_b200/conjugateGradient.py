"""Nonlinear conjugate gradient with the protocol of py-lddmm/conjugateGradient.py.

``cg(opt, verb=True, maxIter=1000, TestGradient=False, epsInit=10.)``
(conjugateGradient.py:33-217): Polak-Ribiere+ directions with a restart every
``restartRate`` (100) iterations, a first trial step, a tiny-step probe on
failure, step halving while it improves, then x1.25 growth while it improves,
stop on |obj - objTry| < 1e-6 (absolute), on |grad| < gradEps or on a bad
direction; eps *= 100 after an accepted step.

The optimiser only ever compares host FP64 scalars: objective values and the
dot products returned by ``opt``; the variables live where ``opt`` keeps them.
"""
import logging

import numpy as np


def cg(opt, verb=True, maxIter=1000, TestGradient=False, epsInit=10.):
    for name in ('getVariable', 'objectiveFun', 'updateTry', 'acceptVarTry', 'getGradient'):
        if not hasattr(opt, name):
            logging.error('Error: required functions are not provided')
            return
    if hasattr(opt, 'startOptim'):
        opt.startOptim()
    gradEps = getattr(opt, 'gradEps', 1.0)
    cgBurnIn = getattr(opt, 'cgBurnIn', -1)
    gradCoeff = getattr(opt, 'gradCoeff', 1.0)
    restartRate = getattr(opt, 'restartRate', 100)

    def dot(g, gs):
        if hasattr(opt, 'dotProduct'):
            return list(opt.dotProduct(g, gs))
        return [float((np.asarray(g) * np.asarray(h)).sum()) for h in gs]

    def copy(g):
        return opt.copyDir(g) if hasattr(opt, 'copyDir') else np.copy(g)

    eps = epsInit
    epsMin = 1e-10
    opt.converged = False
    obj = opt.objectiveFun()
    logging.info('iteration 0: obj = {0: .5f}'.format(obj))
    skipCG = 0
    beta = 0
    grd2 = 0.0
    for it in range(maxIter):
        if it % restartRate == 0:
            skipCG = 1
        if hasattr(opt, 'startOfIteration'):
            opt.startOfIteration()
        grd = opt.getGradient(gradCoeff)
        if TestGradient:
            dirfoo = opt.randomDir() if hasattr(opt, 'randomDir') else np.random.normal(size=np.shape(grd))
            epsfoo = 1e-7
            objfoo = opt.updateTry(dirfoo, epsfoo, obj - 1e10)
            [grdfoo] = dot(grd, [dirfoo])
            # only logged: the difference is formed (and, for values with an
            # error bound, refined) only when the log line is emitted
            if logging.getLogger().isEnabledFor(logging.INFO):
                logging.info('Test Gradient: %.4f %.4f' % ((objfoo - obj) / epsfoo, -grdfoo * gradCoeff))
        if it == 0 or it == cgBurnIn:
            [grdOld2] = dot(grd, [grd])
            grd2 = grdOld2
            grdTry = np.sqrt(max(1e-20, grdOld2))
            oldDir = copy(grd)
            grdOld = copy(grd)
            dir0 = copy(grd)
            beta = 0
        else:
            [grd2, grd12] = dot(grd, [grd, grdOld])
            beta = max(0, (grd2 - grd12) / grdOld2) if skipCG == 0 else 0
            grdOld2 = grd2
            grdTry = np.sqrt(max(1e-20, grd2 + beta * grd12))
            dir0 = opt.addProd(grd, oldDir, beta) if hasattr(opt, 'addProd') else grd + beta * oldDir
            oldDir = copy(dir0)
            grdOld = copy(grd)
        epsSmall = 0.000001 / grdTry
        if hasattr(opt, 'expectTrials'):
            # optional hint (no counterpart in the reference): the tiny-step probe
            # below may follow, so an optimiser that evaluates step sizes in
            # batches can include it; no decision depends on it
            opt.expectTrials(dir0, [eps, epsSmall])
        objTry = opt.updateTry(dir0, eps, obj)
        noUpdate = 0
        if objTry > obj:
            objTry0 = opt.updateTry(dir0, epsSmall, obj)
            if objTry0 > obj:
                if (skipCG == 1) | (beta < 1e-10):
                    logging.info('iteration {0:d}: obj = {1:.5f}, eps = {2:.5f}, beta = {3:.5f}, gradient: {4:.5f}'
                                 .format(it + 1, obj, eps, beta, np.sqrt(grd2)))
                    logging.info('Stopping Gradient Descent: bad direction')
                    break
                else:
                    # conjugateGradient.py:151-154 disables CG and skips the
                    # update only when verb is true; with verb false the
                    # search goes on to the halving loop and accepts objTry
                    if verb:
                        logging.info('Disabling CG: bad direction')
                        skipCG = 1
                        noUpdate = 1
            else:
                while (objTry > obj) and (eps > epsMin):
                    eps = eps / 2
                    objTry = opt.updateTry(dir0, eps, obj)
        if noUpdate == 0:
            while True:
                objTry2 = opt.updateTry(dir0, .5 * eps, objTry)
                if objTry > objTry2:
                    eps = eps / 2
                    objTry = objTry2
                else:
                    break
            while True:
                objTry2 = opt.updateTry(dir0, 1.25 * eps, objTry)
                if objTry > objTry2:
                    eps *= 1.25
                    objTry = objTry2
                else:
                    break
            if np.fabs(obj - objTry) < .000001:
                if (skipCG == 1) | (beta < 1e-10):
                    logging.info('iteration {0:d}: obj = {1:.5f}, eps = {2:.5f}, beta = {3:.5f}, gradient: {4:.5f}'
                                 .format(it + 1, obj, eps, beta, np.sqrt(grd2)))
                    logging.info('Stopping Gradient Descent: small variation')
                    opt.converged = True
                    break
                else:
                    if verb:
                        logging.info('Disabling CG: small variation')
                    skipCG = 1
                    eps = 1.0
            else:
                skipCG = 0
            opt.acceptVarTry()
            obj = objTry
            if verb | (it == maxIter):
                logging.info('iteration {0:d}: obj = {1:.5f}, eps = {2:.5f}, beta = {3:.5f}, gradient: {4:.5f}'
                             .format(it + 1, obj, eps, beta, np.sqrt(grd2)))
            if np.sqrt(grd2) < gradEps:
                logging.info('Stopping Gradient Descent: small gradient')
                opt.converged = True
                break
            eps = 100 * eps
            if hasattr(opt, 'endOfIteration'):
                opt.endOfIteration()
    if hasattr(opt, 'endOptim'):
        opt.endOptim()
    return opt.getVariable()
