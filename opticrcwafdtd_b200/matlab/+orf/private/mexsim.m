function sim = mexsim(sim)
%MEXSIM sim struct in the form the MEX gateway reads: text fields as char
%   (string scalars such as "TE" are objects the C API cannot read), numeric
%   arrays as double, gpuArray data gathered to the host (the gateway passes
%   host arrays to the engine, which copies them to its own device buffers).
for f = {'pol', 'precision'}
    if isfield(sim, f{1}) && isstring(sim.(f{1}))
        sim.(f{1}) = char(sim.(f{1}));
    end
end
for f = {'x', 'y', 'z', 'eps', 'epsX', 'epsZ', 'npml', 'monitors', 'monitorsZ', 'lambdas'}
    if isfield(sim, f{1}) && (isnumeric(sim.(f{1})) || isa(sim.(f{1}), 'gpuArray'))
        sim.(f{1}) = double(gather(sim.(f{1})));
    end
end
if isfield(sim, 'eps') && isstruct(sim.eps)
    for c = {'x', 'y', 'z'}
        if isfield(sim.eps, c{1})
            sim.eps.(c{1}) = double(gather(sim.eps.(c{1})));
        end
    end
end
if isfield(sim, 'source') && isstruct(sim.source)
    for f = {'profile', 'Ea', 'Eb', 'Ha', 'Hb'}
        if isfield(sim.source, f{1}) && (isnumeric(sim.source.(f{1})) || isa(sim.source.(f{1}), 'gpuArray'))
            sim.source.(f{1}) = double(gather(sim.source.(f{1})));
        end
    end
end
end
