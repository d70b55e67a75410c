"""NumPy model of the band-pair H*psi pipeline implemented by the CUDA
kernels in pwdft_develop_b200/csrc/hpsi.cu: two real bands packed as one
complex field, coarse xy planes, z pencils with the Nyquist "+"/"-" slot
unfolding of IP_c2f (src/utility.cpp:3150-3211), fine xy planes with the
local potential and the real-space projectors, and the transposed fold of
IP_f2c (src/utility.cpp:3215-3275).  Used by tests to show the kernel
algorithm equals the reference restatement in exact arithmetic.
"""
import numpy as np
from oracle import pw
def sgn(k,n):  # fft index -> signed (Nyquist +n/2)
    return k if k<=n//2 else k-n
def model_hpsi(T, psi):
    dm=T.dm; n0,n1,n2=dm.numGrid; N0,N1,N2=dm.numGridFine
    nb=psi.shape[0]; out=np.zeros_like(psi)
    ekin_full = 0.5*np.sum(pw.gvec_full(dm)**2,axis=-1)  # (n2,n1,n0)
    fac=dm.vol/dm.ntotFine
    for p in range(0,nb,2):
        a=psi[p].reshape(n2,n1,n0); b=psi[p+1].reshape(n2,n1,n0) if p+1<nb else np.zeros((n2,n1,n0))
        Z=a+1j*b
        # K1: fft x,y per plane
        A=np.fft.fft(np.fft.fft(Z,axis=2),axis=1)
        # K2: fft z, kinetic, unfold+pad z, ifft z (fine)
        X=np.fft.fft(A,axis=0)
        K=ekin_full*X/dm.ntot
        Xs=X/dm.ntot
        B=np.zeros((N2,n1+1,n0+1),complex)
        for ky in range(n1):
            my=sgn(ky,n1); ny=(ky==n1//2)
            for kx in range(n0):
                mx=sgn(kx,n0); nx=(kx==n0//2)
                col=Xs[:,ky,kx]
                if not(ny or nx):
                    cols=[(my,mx,0,1.0)]
                else:
                    cols=[( n1//2 if ny else my, n0//2 if nx else mx, +1, 0.5),
                          (-n1//2 if ny else my,-n0//2 if nx else mx, -1, 0.5)]
                for (sy,sx,sig,w) in cols:
                    f=np.zeros(N2,complex)
                    for kz in range(n2):
                        mz=sgn(kz,n2)
                        if kz==n2//2:
                            if sig==0:
                                f[n2//2]+=0.5*col[kz]; f[N2-n2//2]+=0.5*col[kz]
                            else:
                                f[(sig*n2//2)%N2]+=w*col[kz]
                        else:
                            f[mz%N2]+=w*col[kz]
                    B[:,sy+n1//2,sx+n0//2]=np.fft.ifft(f)*N2
        # K3: per fine plane: pad y, ifft y, pad x, ifft x -> psi_f
        G=np.zeros((N2,N1,n0+1),complex)
        for s in range(n1+1): G[:,(s-n1//2)%N1,:]+=B[:,s,:]
        G=np.fft.ifft(G,axis=1)*N1
        H=np.zeros((N2,N1,N0),complex)
        for s in range(n0+1): H[:,:,(s-n0//2)%N0]+=G[:,:,s]
        psif=np.fft.ifft(H,axis=2)*N0
        pf=psif.reshape(-1)
        upd=pf*T.vtot
        for app in T.pseudo:
            for pp in app:
                w=(pp.val[:,0]@pf[pp.idx])*fac*pp.wgt
                np.add.at(upd,pp.idx,w*pp.val[:,0])
        U=upd.reshape(N2,N1,N0)
        Hx=np.fft.fft(U,axis=2)
        G2=np.zeros((N2,N1,n0+1),complex)
        for s in range(n0+1): G2[:,:,s]=Hx[:,:,(s-n0//2)%N0]
        G2=np.fft.fft(G2,axis=1)
        C=np.zeros((N2,n1+1,n0+1),complex)
        for s in range(n1+1): C[:,s,:]=G2[:,(s-n1//2)%N1,:]
        C/=dm.ntotFine
        # K4: per coarse column: fft z of slot columns, fold, + K, ifft z
        D=np.zeros((n2,n1,n0),complex)
        for ky in range(n1):
            my=sgn(ky,n1); ny=(ky==n1//2)
            for kx in range(n0):
                mx=sgn(kx,n0); nx=(kx==n0//2)
                if not(ny or nx): cols=[(my,mx,0,1.0)]
                else: cols=[( n1//2 if ny else my, n0//2 if nx else mx, +1,0.5),(-n1//2 if ny else my,-n0//2 if nx else mx,-1,0.5)]
                acc=K[:,ky,kx].copy()
                for (sy,sx,sig,w) in cols:
                    f=np.fft.fft(C[:,sy+n1//2,sx+n0//2])
                    for kz in range(n2):
                        mz=sgn(kz,n2)
                        if kz==n2//2:
                            if sig==0: acc[kz]+=0.5*(f[n2//2]+f[N2-n2//2])
                            else: acc[kz]+=w*f[(sig*n2//2)%N2]
                        else: acc[kz]+=w*f[mz%N2]
                D[:,ky,kx]=np.fft.ifft(acc)*n2
        # K5
        R=np.fft.ifft(np.fft.ifft(D,axis=1),axis=2)*n0*n1
        out[p]=R.real.reshape(-1)
        if p+1<nb: out[p+1]=R.imag.reshape(-1)
    return out
