"""dtb: host-side mirror of DiplodocusTransport.jl's explicit Euler path over libdtb.so."""
