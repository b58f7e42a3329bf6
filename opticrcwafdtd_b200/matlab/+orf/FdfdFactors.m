classdef FdfdFactors < handle
    %FDFDFACTORS Device-resident factors of one orf.fdfd2D operator, held
    %   by the MEX gateway under an id and released when the last
    %   reference to this object goes (out.solve and out.adjoint of
    %   orf.fdfd2D hold one).
    properties (SetAccess = private)
        id = 0
    end
    methods
        function obj = FdfdFactors(id)
            obj.id = id;
        end
        function E = solve(obj, J)
            E = orf_fdtd_mex('fdfd2D_solve', obj.id, J, 0);
        end
        function lam = adjoint(obj, g)
            lam = orf_fdtd_mex('fdfd2D_solve', obj.id, g, 1);
        end
        function delete(obj)
            if obj.id > 0
                orf_fdtd_mex('fdfd2D_release', obj.id);
                obj.id = 0;
            end
        end
    end
end
